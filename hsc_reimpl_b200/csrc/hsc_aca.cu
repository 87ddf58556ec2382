// Full-pivot ACA on a 16-CTA thread-block cluster, one cluster per system.
//
// The residual R of the coupling E (qm x a, row-major) lives in distributed
// shared memory: CTA c of the cluster owns columns [c*w, (c+1)*w).  One ACA
// step (core.py:22-50; linear_hsc.cu:248-262) is
//
//   every CTA pushes (max |R|, first row-major index of it, sum R^2) of its
//   slice into every CTA's shared memory and keeps the column of its local
//   argmax (its candidate for u)
//   -- one hardware cluster barrier --
//   every CTA reduces the 16 partials in the same fixed order, picks the
//   pivot (i, j), reads u = R[:, j] from the owning CTA's candidate buffer
//   through DSMEM, forms v = R[i, :] / pivot for its own columns and applies
//   R -= u v^T (rounded as numpy does: multiply, then subtract), while
//   computing the next step's partials.
//
// Partials and candidates are double-buffered, so one barrier per step is
// enough.  Every CTA takes the same decisions from the same bits (the same
// 16 partials, the same candidate column at the same shared-memory offset in
// the owner), so all of them leave the loop at the same step; a last cluster
// barrier keeps each CTA's shared memory alive while the others may read it.  Systems
// whose coupling does not fit 16 CTAs use the cooperative grid version.
#include <cooperative_groups.h>

#include <cfloat>

#include "hsc_check.cuh"
#include "hsc_setup.cuh"

namespace cg = cooperative_groups;

namespace hsc {

namespace {

constexpr int kAcaCluster = 16;
constexpr int kAcaThreads = 1024;
constexpr int kAcaWarps = kAcaThreads / 32;

struct Part {
    double vmax;
    long long idx;
    double sum;
    double pad;
};

__device__ __forceinline__ void better_into(double& v, long long& i, double qv, long long qi) {
    if (qv > v || (qv == v && qi < i)) { v = qv; i = qi; }
}

// the same order on a CTA-local row-major index (r * nl + c): within one CTA's
// column slice it orders entries exactly as the global row-major index does
__device__ __forceinline__ void better_into32(double& v, int& i, double qv, int qi) {
    if (qv > v || (qv == v && qi < i)) { v = qv; i = qi; }
}

__device__ __forceinline__ void warp_best32(double& v, int& i, double& s) {
    for (int o = 16; o > 0; o >>= 1) {
        const double qv = __shfl_xor_sync(0xffffffffu, v, o);
        const int qi = __shfl_xor_sync(0xffffffffu, i, o);
        s += __shfl_xor_sync(0xffffffffu, s, o);
        better_into32(v, i, qv, qi);
    }
}

__device__ __forceinline__ void warp_best(double& v, long long& i, double& s, int width) {
    for (int o = width / 2; o > 0; o >>= 1) {
        const double qv = __shfl_xor_sync(0xffffffffu, v, o);
        const long long qi = __shfl_xor_sync(0xffffffffu, i, o);
        s += __shfl_xor_sync(0xffffffffu, s, o);
        better_into(v, i, qv, qi);
    }
}

__global__ void __launch_bounds__(kAcaThreads, 1) aca_cluster_kernel(const AcaSys* sys) {
    cg::cluster_group cl = cg::this_cluster();
    const AcaSys P = sys[blockIdx.x / kAcaCluster];
    if (cl.num_blocks() != kAcaCluster) {  // launched without the 16-CTA cluster: refuse, uniformly
        if (threadIdx.x == 0 && blockIdx.x % kAcaCluster == 0) { *P.rank = 0; *P.err = -1.0; }
        return;
    }
    const int cr = (int)cl.block_rank();
    const int m = P.m, nc = P.nc;
    const int w = (nc + kAcaCluster - 1) / kAcaCluster;
    const int c0 = min(nc, cr * w), c1 = min(nc, c0 + w), nl = c1 - c0;
    const long long total = (long long)m * nc;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    extern __shared__ double sm[];
    // the same layout in every CTA of the cluster (offsets must not depend on
    // this CTA's own width nl): DSMEM maps an offset into the peer's memory
    double* R = sm;                 // m x nl, row-major, in an m x w region
    double* cand = R + m * w;       // 2 x m candidate columns
    double* u = cand + 2 * m;       // m
    double* v = u + m;              // nl <= w
    __shared__ Part part[2];
    __shared__ Part parts[2][kAcaCluster];  // every CTA's step partial, pushed by its owner
    __shared__ Part s_w[kAcaWarps];
    __shared__ double s_sc[2];
    __shared__ long long s_si;
    __shared__ int s_bl;  // this CTA's local argmax (publish)

    for (int r = warp; r < m; r += kAcaWarps)
        for (int c = lane; c < nl; c += 32)
            if (HSC_IN(c0 + c < nc && r * nl + c < m * nl, 102, c0 + c)) R[r * nl + c] = P.E[(size_t)r * nc + c0 + c];
    cl.sync();  // every CTA of the cluster has started before the first push into its shared memory

    // local (max, idx, sum) of the slice -> part[slot] (global index); candidate column -> cand[slot].
    // The argmax runs on the CTA-local index; kNone marks an empty slice.
    constexpr int kNone = 0x7fffffff;
    auto publish = [&](int slot, double ls, double lv, int li) {
        warp_best32(lv, li, ls);
        if (lane == 0) { s_w[warp].vmax = lv; s_w[warp].idx = li; s_w[warp].sum = ls; }
        __syncthreads();
        if (warp == 0) {
            // the warp partials in a fixed tree order (the same bits in every run)
            double bv = -1.0, bs = 0.0;
            int bi = kNone;
            if (lane < kAcaWarps) { bv = s_w[lane].vmax; bi = (int)s_w[lane].idx; bs = s_w[lane].sum; }
            warp_best32(bv, bi, bs);
            const long long gi = bi == kNone ? total : (long long)(bi / nl) * nc + c0 + bi % nl;
            const Part pt{bv, gi, bs, 0.0};
            if (lane == 0) { part[slot] = pt; s_bl = bi; }
            // push it to every CTA of the cluster (the cluster barrier publishes it)
            if (lane < kAcaCluster) *cl.map_shared_rank(&parts[slot][cr], lane) = pt;
        }
        __syncthreads();
        const int bl = s_bl;
        if (bl != kNone) {
            const int jl = bl % nl;
            for (int r = tid; r < m; r += kAcaThreads)
                if (HSC_IN(jl >= 0 && jl < nl, 103, jl)) cand[slot * m + r] = R[r * nl + jl];
        }
    };
    {
        double ls = 0.0, lv = -1.0;
        int li = kNone;
        for (int r = warp; r < m; r += kAcaWarps)
            for (int c = lane; c < nl; c += 32) {
                const double x = R[r * nl + c];
                ls += x * x;
                better_into32(lv, li, fabs(x), r * nl + c);
            }
        publish(0, ls, lv, li);
    }
    double scale = 0.0, residual = 0.0;
    int k = 0;
    for (;; ++k) {
        const int slot = k & 1;
        cl.sync();
        if (warp == 0) {
            double pv = -1.0, ps = 0.0;
            long long pi = total;
            if (lane < kAcaCluster && HSC_IN(lane < (int)cl.num_blocks(), 109, lane)) {
                const Part& rp = parts[slot][lane];
                pv = rp.vmax; pi = rp.idx; ps = rp.sum;
            }
            warp_best(pv, pi, ps, 32);
            if (lane == 0) { s_sc[0] = ps; s_sc[1] = pv; s_si = pi; }
        }
        __syncthreads();
        const double gsum = s_sc[0];
        const long long gi = s_si;
        if (k == 0) {
            scale = sqrt(gsum);
            residual = scale > 0 ? 1.0 : 0.0;
        } else {
            residual = sqrt(gsum) / scale;
        }
        if (cr == 0 && tid == 0) P.hist[k] = residual;
        if (!(residual > P.rtol) || k >= P.cap || gi >= total) break;
        const int i = (int)(gi / nc), j = (int)(gi - (long long)i * nc);
        const int owner = j / w;
        const bool own_ok = HSC_IN(owner >= 0 && owner < (int)cl.num_blocks() && i < m, 110, owner);
        const double* rc = cl.map_shared_rank(cand + slot * m, own_ok ? owner : 0);
        for (int r = tid; r < m; r += kAcaThreads) u[r] = own_ok ? rc[r] : 0.0;
        __syncthreads();
        const double pivot = u[i];
        if (!(fabs(pivot) > DBL_EPSILON * fmax(scale, DBL_MIN))) break;
        for (int c = tid; c < nl; c += kAcaThreads) v[c] = R[i * nl + c] / pivot;
        __syncthreads();
        if (cr == 0)
            for (int r = tid; r < m; r += kAcaThreads)
                if (HSC_IN(k < P.cap, 106, k)) P.U[(size_t)k * m + r] = u[r];
        for (int c = tid; c < nl; c += kAcaThreads)
            if (HSC_IN(k < P.cap && c0 + c < nc, 107, k)) P.V[(size_t)k * nc + c0 + c] = v[c];
        double ls = 0.0, lv = -1.0;
        int li = kNone;
        for (int r = warp; r < m; r += kAcaWarps) {
            const double ur = u[r];
            for (int c = lane; c < nl; c += 32) {
                const double x = __dsub_rn(R[r * nl + c], __dmul_rn(ur, v[c]));  // numpy: R - outer(u, v)
                R[r * nl + c] = x;
                ls += x * x;
                better_into32(lv, li, fabs(x), r * nl + c);
            }
        }
        publish(slot ^ 1, ls, lv, li);
    }
    cl.sync();
    if (cr == 0 && tid == 0) {
        *P.rank = k;
        *P.err = residual;
    }
}

}  // namespace

size_t aca_cluster_smem_doubles(int m, int nc) {
    const int w = (nc + kAcaCluster - 1) / kAcaCluster;
    return (size_t)m * w + 3 * (size_t)m + w + 2;
}

bool aca_cluster_fits(int m, int nc) {
    return aca_cluster_smem_doubles(m, nc) * sizeof(double) <= 200 * 1024;
}

cudaError_t launch_aca_cluster(const AcaSys* d_sys, int nsys, size_t smem_doubles, cudaStream_t st) {
    if (nsys <= 0) return cudaSuccess;
    const size_t bytes = smem_doubles * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(aca_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(aca_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nsys * kAcaCluster);
    cfg.blockDim = dim3(kAcaThreads);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kAcaCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    count_launch();
    return cudaLaunchKernelEx(&cfg, aca_cluster_kernel, d_sys);
}

void read_fail_aca(long long* out) { hsc_read_fail(out); }

int aca_cluster_supported(size_t smem_doubles) {
    cudaError_t e = cudaFuncSetAttribute(aca_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return 0;
    e = cudaFuncSetAttribute(aca_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(smem_doubles * sizeof(double)));
    if (e != cudaSuccess) return 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kAcaCluster);
    cfg.blockDim = dim3(kAcaThreads);
    cfg.dynamicSmemBytes = smem_doubles * sizeof(double);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kAcaCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, aca_cluster_kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

}  // namespace hsc
