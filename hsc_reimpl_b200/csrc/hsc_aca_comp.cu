// Full-pivot ACA by coupling component, merged into the global pivot order.
//
// The coupling E (qm x a) is block-structured: the rows of an affine body are
// nonzero only at the columns of the FEM nodes it touches, so after ordering
// rows by body and columns by node, E is block diagonal over the coupling
// components (bodies joined through shared nodes).  A full-pivot ACA step
// (core.py:22-50, linear_hsc.cu:248-262) picks the global argmax |R|, and the
// update R -= u v^T only touches the pivot's component (u lives on its rows, v
// on its columns).  So each component's pivots come in the same order whether
// the ACA runs on E or on that component alone, and the global sequence is the
// merge of the components' sequences by pivot magnitude (ties to the first
// row-major index, as argmax takes them).
//
// Here every component runs its own ACA in one CTA (its residual block in
// shared memory when it fits), all components at once; one thread then merges
// the sequences, applying the global stop rules (rank cap, relative Frobenius
// residual from the components' sums of squares, zero-pivot guard), and the
// columns are scattered into U and V in merged order.  The result is the
// global ACA's factorization: the same pivots, the same columns in the same
// order, each entry computed with the same operations (R - u v rounded as
// numpy rounds it).  A coupling of vehicle size (144 x 2,976, rank 96) takes
// 96 sequential steps globally; by component it is 12 steps per CTA.
#include <cfloat>
#include <climits>

#include "hsc_check.cuh"
#include "hsc_setup.cuh"

namespace hsc {

namespace {

constexpr int kCompThreads = 512;
constexpr int kCompWarps = kCompThreads / 32;

// CTA-wide (max |.|, first local row-major index, sum of squares) of the residual
// block.  Rows and columns of a component ascend, so the local row-major order is
// the global one restricted to the block: the first local maximum is the global
// argmax's choice among the block's entries.
__device__ void block_stats(const double* R, int n, double& vmax, int& imax, double& sum) {
    __shared__ double s_v[kCompWarps], s_s[kCompWarps];
    __shared__ int s_i[kCompWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double lv = -1.0, ls = 0.0;
    int li = INT_MAX;
    for (int e = threadIdx.x; e < n; e += kCompThreads) {
        const double x = R[e];
        ls += x * x;
        const double ax = fabs(x);
        if (ax > lv) { lv = ax; li = e; }     // a thread's entries ascend: ties keep the first
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double qv = __shfl_xor_sync(0xffffffffu, lv, o);
        const int qi = __shfl_xor_sync(0xffffffffu, li, o);
        ls += __shfl_xor_sync(0xffffffffu, ls, o);
        if (qv > lv || (qv == lv && qi < li)) { lv = qv; li = qi; }
    }
    if (lane == 0) { s_v[warp] = lv; s_i[warp] = li; s_s[warp] = ls; }
    __syncthreads();
    if (warp == 0) {
        lv = lane < kCompWarps ? s_v[lane] : -1.0;
        li = lane < kCompWarps ? s_i[lane] : INT_MAX;
        ls = lane < kCompWarps ? s_s[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            const double qv = __shfl_xor_sync(0xffffffffu, lv, o);
            const int qi = __shfl_xor_sync(0xffffffffu, li, o);
            ls += __shfl_xor_sync(0xffffffffu, ls, o);
            if (qv > lv || (qv == lv && qi < li)) { lv = qv; li = qi; }
        }
        if (lane == 0) { s_v[0] = lv; s_i[0] = li; s_s[0] = ls; }
    }
    __syncthreads();
    vmax = s_v[0];
    imax = s_i[0];
    sum = s_s[0];
    __syncthreads();
}

// sum of squares of E (the scale of the zero-pivot guard and of the residuals)
__global__ void e_sumsq_kernel(const double* E, long long n, double* out) {
    __shared__ double s[32];
    double a = 0.0;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) a += E[e] * E[e];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
        *out = t;
    }
}

__global__ void __launch_bounds__(kCompThreads) aca_comp_kernel(AcaComp p) {
    const int g = blockIdx.x;
    const int r0 = p.row_ptr[g], mr = p.row_ptr[g + 1] - r0;
    const int c0 = p.col_ptr[g], nc = p.col_ptr[g + 1] - c0;
    const int* rows = p.rows + r0;
    const int* cols = p.cols + c0;
    const int steps_max = min(min(mr, nc), p.kmax);
    extern __shared__ double sm[];
    const bool in_smem = (size_t)mr * nc <= (size_t)p.smem_doubles;
    double* R = in_smem ? sm : p.Rscratch + p.r_off[g];
    __shared__ double s_u[256];          // u = R[:, j]; the host admits components of at most 256 rows
    __shared__ double s_piv;
    __shared__ int s_i, s_j;
    for (int e = threadIdx.x; e < mr * nc; e += kCompThreads) {
        const int r = e / nc, c = e - r * nc;
        R[e] = p.E[(size_t)rows[r] * p.a + cols[c]];
    }
    __syncthreads();
    const double scale = sqrt(*p.esumsq);
    double vmax, sum;
    int imax;
    block_stats(R, mr * nc, vmax, imax, sum);
    double* piv_abs = p.piv_abs + p.s_off[g];
    long long* piv_idx = p.piv_idx + p.s_off[g];
    double* sums = p.sums + p.s_off[g] + g;   // steps_max + 1 entries per component
    double* Ug = p.Ug + p.u_off[g];            // mr x steps, one column per step
    double* Vg = p.Vg + p.v_off[g];            // nc x steps
    int s = 0;
    for (; s < steps_max; ++s) {
        if (threadIdx.x == 0) sums[s] = sum;
        if (!(vmax > DBL_EPSILON * fmax(scale, DBL_MIN)) || imax == INT_MAX) break;  // zero-pivot guard
        if (threadIdx.x == 0) {
            const int li = imax / nc, lj = imax - li * nc;
            piv_abs[s] = vmax;
            piv_idx[s] = (long long)rows[li] * p.a + cols[lj];  // the global row-major index, for the merge
            s_i = li;
            s_j = lj;
        }
        __syncthreads();
        const int i = s_i, j = s_j;
        for (int r = threadIdx.x; r < mr; r += kCompThreads) s_u[r] = R[(size_t)r * nc + j];
        if (threadIdx.x == 0) s_piv = R[(size_t)i * nc + j];
        __syncthreads();
        const double pivot = s_piv;
        for (int r = threadIdx.x; r < mr; r += kCompThreads) Ug[(size_t)s * mr + r] = s_u[r];
        // v = R[i, :] / pivot, then R -= u v^T (the product rounded, then the difference: numpy's order)
        for (int c = threadIdx.x; c < nc; c += kCompThreads) Vg[(size_t)s * nc + c] = R[(size_t)i * nc + c] / pivot;
        __syncthreads();
        for (int e = threadIdx.x; e < mr * nc; e += kCompThreads) {
            const int r = e / nc, c = e - r * nc;
            R[e] = __dsub_rn(R[e], __dmul_rn(s_u[r], Vg[(size_t)s * nc + c]));
        }
        __syncthreads();
        block_stats(R, mr * nc, vmax, imax, sum);
    }
    if (threadIdx.x == 0) {
        p.nsteps[g] = s;
        sums[s] = sum;
    }
}

// one thread: merge the components' pivot sequences into the global order and
// apply the global stop rules; order[t] = (component, its step)
__global__ void aca_merge_kernel(AcaComp p) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double scale = sqrt(*p.esumsq);
    int t = 0;
    for (int g = 0; g < p.ncomp; ++g) p.cur[g] = 0;
    for (;; ++t) {
        double rs = 0.0;
        for (int g = 0; g < p.ncomp; ++g) rs += p.sums[p.s_off[g] + g + p.cur[g]];
        const double residual = t == 0 ? (scale > 0 ? 1.0 : 0.0) : sqrt(rs) / scale;
        p.hist[t] = residual;
        if (!(residual > p.rtol) || t >= p.kmax) break;
        int best = -1;
        for (int g = 0; g < p.ncomp; ++g) {
            if (p.cur[g] >= p.nsteps[g]) continue;
            if (best < 0) { best = g; continue; }
            const double v = p.piv_abs[p.s_off[g] + p.cur[g]];
            const long long i = p.piv_idx[p.s_off[g] + p.cur[g]];
            const double bv = p.piv_abs[p.s_off[best] + p.cur[best]];
            const long long bi = p.piv_idx[p.s_off[best] + p.cur[best]];
            if (v > bv || (v == bv && i < bi)) best = g;
        }
        if (best < 0) break;  // every component is exhausted: the guard stops the global ACA too
        p.order[2 * t] = best;
        p.order[2 * t + 1] = p.cur[best]++;
    }
    *p.rank = t;
    *p.err = p.hist[t];
}

// U[:, t] and V[:, t] from the components' columns (zero elsewhere), t < kmax
__global__ void aca_scatter_kernel(AcaComp p) {
    const int t = blockIdx.x;
    const int k = *p.rank;
    double* Ut = p.U + (size_t)t * p.qm;
    double* Vt = p.V + (size_t)t * p.a;
    for (int r = threadIdx.x; r < p.qm; r += blockDim.x) Ut[r] = 0.0;
    for (int c = threadIdx.x; c < p.a; c += blockDim.x) Vt[c] = 0.0;
    if (t >= k) return;
    __syncthreads();
    const int g = p.order[2 * t], s = p.order[2 * t + 1];
    const int r0 = p.row_ptr[g], mr = p.row_ptr[g + 1] - r0;
    const int c0 = p.col_ptr[g], nc = p.col_ptr[g + 1] - c0;
    const double* Ug = p.Ug + p.u_off[g] + (size_t)s * mr;
    const double* Vg = p.Vg + p.v_off[g] + (size_t)s * nc;
    for (int r = threadIdx.x; r < mr; r += blockDim.x) Ut[p.rows[r0 + r]] = Ug[r];
    for (int c = threadIdx.x; c < nc; c += blockDim.x) Vt[p.cols[c0 + c]] = Vg[c];
}

}  // namespace

size_t aca_comp_smem_doubles() { return (220 * 1024) / sizeof(double); }

cudaError_t launch_aca_comp(const AcaComp& p, cudaStream_t st) {
    count_launch();
    e_sumsq_kernel<<<1, 1024, 0, st>>>(p.E, (long long)p.qm * p.a, p.esumsq);
    if (p.ncomp > 0) {
        const size_t smem = sizeof(double) * (size_t)p.smem_doubles;
        cudaError_t e = cudaFuncSetAttribute(aca_comp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        count_launch();
        aca_comp_kernel<<<p.ncomp, kCompThreads, smem, st>>>(p);
    }
    count_launch();
    aca_merge_kernel<<<1, 32, 0, st>>>(p);
    count_launch();
    aca_scatter_kernel<<<p.kmax, 256, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace hsc
