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
// shared memory when it fits), all components at once, until its residual
// vanishes; one warp then merges the sequences, applying the global stop rules
// (rank cap, relative Frobenius residual from the components' sums of squares,
// zero-pivot guard against |E|_F, which is the root of the sum of the
// components' initial sums since E vanishes outside them), and the columns are
// scattered into U and V in merged order.  The result is the
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

constexpr int kCompThreads = 1024;
constexpr int kCompWarps = kCompThreads / 32;

// CTA-wide (max |.|, first local row-major index, sum of squares) from each thread's partial
// (lv, li, ls).  Rows and columns of a component ascend, so the local row-major order is the
// global one restricted to the block: the first local maximum is the global argmax's choice
// among the block's entries (the maximum and its first index do not depend on the order the
// entries were visited in).
__device__ void block_reduce(double lv, int li, double ls, double& vmax, int& imax, double& sum) {
    __shared__ double s_v[kCompWarps], s_s[kCompWarps];
    __shared__ int s_i[kCompWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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

__device__ __forceinline__ void stat_add(double x, int e, double& lv, int& li, double& ls) {
    ls += x * x;
    const double ax = fabs(x);
    if (ax > lv || (ax == lv && e < li)) { lv = ax; li = e; }
}

// one CTA per coupling component: the full-pivot ACA of its block of E.  Thread t owns the
// columns t, t + kCompThreads, ... of the block (all rows), so a step is one pass: v = R[i, :] /
// pivot and R -= u v^T on its columns, folding the next step's statistics in.
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
    double lv = -1.0, ls = 0.0;
    int li = INT_MAX;
    for (int c = threadIdx.x; c < nc; c += kCompThreads) {
        const int gc = cols[c];
        for (int r = 0; r < mr; ++r) {
            const double x = p.E[(size_t)rows[r] * p.a + gc];
            R[(size_t)r * nc + c] = x;
            stat_add(x, r * nc + c, lv, li, ls);
        }
    }
    double vmax, sum;
    int imax;
    block_reduce(lv, li, ls, vmax, imax, sum);  // synchronises: R is complete
    double* piv_abs = p.piv_abs + p.s_off[g];
    long long* piv_idx = p.piv_idx + p.s_off[g];
    double* sums = p.sums + p.s_off[g] + g;   // steps_max + 1 entries per component
    double* Ug = p.Ug + p.u_off[g];            // mr x steps, one column per step
    double* Vg = p.Vg + p.v_off[g];            // nc x steps
    int s = 0;
    for (; s < steps_max; ++s) {
        if (threadIdx.x == 0) sums[s] = sum;
        if (!(vmax > 0.0) || imax == INT_MAX) break;  // the residual vanished (the merge applies the guard)
        const int i = imax / nc, j = imax - i * nc;
        if (threadIdx.x == 0) {
            piv_abs[s] = vmax;
            piv_idx[s] = (long long)rows[i] * p.a + cols[j];  // the global row-major index, for the merge
            s_piv = R[(size_t)i * nc + j];
        }
        for (int r = threadIdx.x; r < mr; r += kCompThreads) {
            const double u = R[(size_t)r * nc + j];
            s_u[r] = u;
            Ug[(size_t)s * mr + r] = u;
        }
        __syncthreads();
        const double pivot = s_piv;
        // v = R[i, :] / pivot, then R -= u v^T (the product rounded, then the difference: numpy's order)
        double* Vs = Vg + (size_t)s * nc;
        lv = -1.0; ls = 0.0; li = INT_MAX;
        for (int c = threadIdx.x; c < nc; c += kCompThreads) {
            const double vc = R[(size_t)i * nc + c] / pivot;
            Vs[c] = vc;
            for (int r = 0; r < mr; ++r) {
                const double x = __dsub_rn(R[(size_t)r * nc + c], __dmul_rn(s_u[r], vc));
                R[(size_t)r * nc + c] = x;
                stat_add(x, r * nc + c, lv, li, ls);
            }
        }
        block_reduce(lv, li, ls, vmax, imax, sum);
    }
    if (threadIdx.x == 0) {
        p.nsteps[g] = s;
        sums[s] = sum;
    }
}

constexpr int kMergePer = 8;  // components per lane in the warp merge (256 / 32)

// The greedy picks of the merge, by one warp: lane l follows the cursors of components l + 32 i
// (i < PER); each pick is the largest current pivot (ties to the first row-major index), until the
// rank cap, exhaustion or the zero-pivot guard.  Returns the number of picks.
template <int PER>
__device__ int merge_picks(const AcaComp& p, int G, const double* pa, const long long* pi, const int* so,
                           const int* nst, int* comp, double guard) {
    const int lane = threadIdx.x & 31;
    int span = 1;                                                // butterfly rounds cover min(G, 32) lanes
    while (span < min(G, 32)) span <<= 1;
    int cur[PER], off[PER], lim[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int c = lane + 32 * i;
        cur[i] = 0;
        off[i] = c < G ? so[c] : 0;
        lim[i] = c < G ? nst[c] : 0;
    }
    int t = 0;
    for (; t < p.kmax; ++t) {
        double bv = -1.0;
        long long bi = LLONG_MAX;
        int bc = -1, bs = 0;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            if (cur[i] < lim[i]) {
                const double v = pa[off[i] + cur[i]];
                const long long ix = pi[off[i] + cur[i]];
                if (v > bv || (v == bv && ix < bi)) { bv = v; bi = ix; bc = lane + 32 * i; bs = cur[i]; }
            }
        }
        for (int o = span >> 1; o > 0; o >>= 1) {
            const double qv = __shfl_xor_sync(0xffffffffu, bv, o);
            const long long qi = __shfl_xor_sync(0xffffffffu, bi, o);
            const int qc = __shfl_xor_sync(0xffffffffu, bc, o), qs = __shfl_xor_sync(0xffffffffu, bs, o);
            if (qv > bv || (qv == bv && qi < bi)) { bv = qv; bi = qi; bc = qc; bs = qs; }
        }
        bv = __shfl_sync(0xffffffffu, bv, 0);
        bc = __shfl_sync(0xffffffffu, bc, 0);
        bs = __shfl_sync(0xffffffffu, bs, 0);
        if (bc < 0 || !(bv > guard)) break;  // exhausted, or the zero-pivot guard on the global argmax
        if (lane == 0) { p.order[2 * t] = bc; p.order[2 * t + 1] = bs; comp[t] = bc; }
        if ((bc & 31) == lane) {
#pragma unroll
            for (int i = 0; i < PER; ++i)
                if (i == (bc >> 5)) ++cur[i];
        }
    }
    return t;
}

// Merge the components' pivot sequences into the global order and apply the global stop rules;
// order[t] = (component, its step).  The order depends on the pivots alone, so one warp first
// picks greedily (the largest current pivot, ties to the first row-major index) until the rank
// cap, exhaustion or the zero-pivot guard stops it (T picks); then every thread takes one t <= T
// and forms the relative residual before pick t from the components' sums of squares (summed in
// component order), and the rank is the first t whose residual reaches rtol, else T.  The step
// records are staged in shared memory first.
__global__ void __launch_bounds__(256) aca_merge_kernel(AcaComp p) {
    extern __shared__ double msm[];
    const int G = p.ncomp, ns = p.stot, K1 = p.kmax + 1;
    double* pa = msm;                                            // ns
    double* su = pa + ns;                                        // ns + G
    double* tab = su + ns + G;                                   // K1 x G: sums before each pick
    double* res = tab + (size_t)K1 * G;                          // K1
    long long* pi = reinterpret_cast<long long*>(res + K1);      // ns
    int* so = reinterpret_cast<int*>(pi + ns);                   // G
    int* nst = so + G;                                           // G
    int* comp = nst + G;                                         // K1: component of each pick
    __shared__ int s_T, s_rank;
    __shared__ double s_scale;
    for (int e = threadIdx.x; e < ns; e += blockDim.x) { pa[e] = p.piv_abs[e]; pi[e] = p.piv_idx[e]; }
    for (int e = threadIdx.x; e < ns + G; e += blockDim.x) su[e] = p.sums[e];
    for (int e = threadIdx.x; e < G; e += blockDim.x) { so[e] = p.s_off[e]; nst[e] = p.nsteps[e]; }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double e2 = 0.0;
        for (int c = lane; c < G; c += 32) e2 += su[so[c] + c];
        for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
        const double scale = sqrt(e2);
        const double guard = DBL_EPSILON * fmax(scale, DBL_MIN);
        const int T = G <= 32 ? merge_picks<1>(p, G, pa, pi, so, nst, comp, guard)
                              : merge_picks<kMergePer>(p, G, pa, pi, so, nst, comp, guard);
        if (lane == 0) { s_T = T; s_scale = scale; }
    }
    __syncthreads();
    const int T = s_T;
    const double scale = s_scale;
    // tab[t][c] = component c's residual sum of squares before pick t
    for (int c = threadIdx.x; c < G; c += blockDim.x) {
        int n = 0;
        for (int t = 0; t <= T; ++t) {
            tab[(size_t)t * G + c] = su[so[c] + c + n];
            if (t < T && comp[t] == c) ++n;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t <= T; t += blockDim.x) {
        double rs = 0.0;
        for (int c = 0; c < G; ++c) rs += tab[(size_t)t * G + c];
        res[t] = t == 0 ? (scale > 0 ? 1.0 : 0.0) : sqrt(rs) / scale;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int r = 0;
        while (r < T && res[r] > p.rtol) ++r;
        s_rank = r;
        *p.rank = r;
        *p.err = res[r];
    }
    __syncthreads();
    for (int t = threadIdx.x; t <= s_rank; t += blockDim.x) p.hist[t] = res[t];
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

size_t aca_merge_smem_bytes(int ncomp, int stot, int kmax) {
    const size_t k1 = (size_t)kmax + 1;
    return sizeof(double) * (3 * (size_t)stot + ncomp + k1 * ncomp + k1) + sizeof(int) * (2 * (size_t)ncomp + k1);
}

bool aca_merge_fits(int ncomp, int stot, int kmax) {
    return ncomp <= 32 * kMergePer && aca_merge_smem_bytes(ncomp, stot, kmax) <= 200 * 1024;
}

cudaError_t launch_aca_comp(const AcaComp& p, cudaStream_t st) {
    if (p.ncomp > 0) {
        const size_t smem = sizeof(double) * (size_t)p.smem_doubles;
        cudaError_t e = cudaFuncSetAttribute(aca_comp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        count_launch();
        aca_comp_kernel<<<p.ncomp, kCompThreads, smem, st>>>(p);
    }
    const size_t msmem = aca_merge_smem_bytes(p.ncomp, p.stot, p.kmax);
    cudaError_t e = cudaFuncSetAttribute(aca_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)msmem);
    if (e != cudaSuccess) return e;
    count_launch();
    aca_merge_kernel<<<1, 256, msmem, st>>>(p);
    count_launch();
    aca_scatter_kernel<<<p.kmax, 256, 0, st>>>(p);
    return cudaPeekAtLastError();
}

}  // namespace hsc
