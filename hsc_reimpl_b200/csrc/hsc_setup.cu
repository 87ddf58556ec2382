// Numeric setup kernels of one HSC solve (everything the reference does in
// LinearHSC::setup, linear_hsc.cu:195-304, moved onto the GPU):
//   * pattern hash of the BCOO indices (detects a changed pattern behind the
//     same pointers);
//   * BCOO (one triangle, column-major 3x3) -> full row-owner BSR planes;
//   * FEM 3x3 diagonal inverses with the det > 0 check (linear_hsc.cu:70-80);
//   * dense A (qm x qm) and coupling E (qm x a) over the sorted active FEM
//     dofs (linear_hsc.cu:216-247);
//   * full-pivot ACA of E as one cooperative kernel (core.py:22-50);
//   * small dense FP64 algebra for the ABD inverse and the reduced core
//     (Cholesky, triangular solves, tiled GEMM, LDL^T);
//   * right-hand side, back-substitution and the full-system residual.
#include "hsc_check.cuh"
#include "hsc_setup.cuh"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cfloat>

namespace hsc {

// kernels launched by this library (for the launch count a benchmark reports)
static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
// HSC_SYNC_CHECK=1 (debugging, no graph capture): synchronise after every
// launch of this library and name the first launch that left an error
void debug_sync(const char* what) {
    static int on = -1;
    if (on < 0) {
        const char* e = std::getenv("HSC_SYNC_CHECK");
        on = (e && *e && *e != '0') ? 1 : 0;
    }
    if (!on) return;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) std::fprintf(stderr, "HSC_SYNC_CHECK: %s after %s\n", cudaGetErrorString(e), what);
}
#define HSC_COUNTED(...)      \
    do {                      \
        ::hsc::count_launch(); \
        __VA_ARGS__;          \
        ::hsc::debug_sync(#__VA_ARGS__); \
    } while (0)

namespace {

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double bsum(double v) {
    __shared__ double s[32];
    v = wsum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) s[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (warp == 0) {
        t = lane < nw ? s[lane] : 0.0;
        t = wsum(t);
    }
    return t;  // valid in thread 0
}

// ---------------------------------------------------------------------------
__global__ void pattern_hash_kernel(const int* rows, const int* cols, long long nnzb,
                                    unsigned long long* out) {
    unsigned long long h = 0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nnzb;
         t += (long long)gridDim.x * blockDim.x) {
        unsigned long long v = ((unsigned long long)(unsigned)rows[t] << 32) | (unsigned)cols[t];
        v ^= (unsigned long long)(t + 1) * 0x9E3779B97F4A7C15ull;
        v ^= v >> 31; v *= 0xBF58476D1CE4E5B9ull; v ^= v >> 29;
        h += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, h);
}

// BCOO entry -> full BSR planes: FP64 always, plus an FP32 and/or a BF16 copy
__global__ void fill_bsr_kernel(const int* src, const double* values, int nnz, double* v64, float* vf,
                                __nv_bfloat16* vb) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const int packed = src[k];
    const long long t = packed >> 1;
    const int tr = packed & 1;
    const double* B = values + 9 * t;  // B(r, c) = B[r + 3 c]
#pragma unroll
    for (int rr = 0; rr < 3; ++rr)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
            const double v = tr ? B[cc + 3 * rr] : B[rr + 3 * cc];
            const size_t o = (size_t)(3 * rr + cc) * nnz + k;
            v64[o] = v;
            if (vf) vf[o] = (float)v;
            if (vb) vb[o] = __float2bfloat16_rn((float)v);
        }
}

template <class DT>
__global__ void dinv_kernel(const int* diag_pos, const double* v64, int nnz, int n, DT* dinv, int* bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = diag_pos[i];
    double b[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) b[e] = v64[(size_t)e * nnz + k];
    // adjugate / det
    const double c00 = b[4] * b[8] - b[5] * b[7];
    const double c01 = b[5] * b[6] - b[3] * b[8];
    const double c02 = b[3] * b[7] - b[4] * b[6];
    const double det = b[0] * c00 + b[1] * c01 + b[2] * c02;
    double inv[9];
    if (!(det > 0.0) || !isfinite(det)) {
        atomicAdd(bad, 1);
#pragma unroll
        for (int e = 0; e < 9; ++e) inv[e] = 0.0;
    } else {
        const double id = 1.0 / det;
        inv[0] = c00 * id;
        inv[1] = (b[2] * b[7] - b[1] * b[8]) * id;
        inv[2] = (b[1] * b[5] - b[2] * b[4]) * id;
        inv[3] = c01 * id;
        inv[4] = (b[0] * b[8] - b[2] * b[6]) * id;
        inv[5] = (b[2] * b[3] - b[0] * b[5]) * id;
        inv[6] = c02 * id;
        inv[7] = (b[1] * b[6] - b[0] * b[7]) * id;
        inv[8] = (b[0] * b[4] - b[1] * b[3]) * id;
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) dinv[(size_t)e * n + i] = (DT)inv[e];
}

__global__ void extract_A_kernel(const int* list, int count, const double* values, int qm, double* A) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const long long t = list[3 * e];
    const int ar = list[3 * e + 1], ac = list[3 * e + 2];
    const double* B = values + 9 * t;
    for (int rr = 0; rr < 3; ++rr)
        for (int cc = 0; cc < 3; ++cc) {
            const double v = B[rr + 3 * cc];
            A[(size_t)(3 * ar + rr) * qm + 3 * ac + cc] = v;
            if (ar != ac) A[(size_t)(3 * ac + cc) * qm + 3 * ar + rr] = v;
        }
}

__global__ void extract_E_kernel(const int* list, int count, const double* values, int a, double* E,
                                 int* node_nz) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const long long t = list[4 * e];
    const int q = list[4 * e + 1], an = list[4 * e + 2], orient = list[4 * e + 3];
    const double* B = values + 9 * t;
    double sq = 0.0;
    for (int rr = 0; rr < 3; ++rr)
        for (int cc = 0; cc < 3; ++cc) {
            const double v = orient ? B[cc + 3 * rr] : B[rr + 3 * cc];
            E[(size_t)(3 * q + rr) * a + 3 * an + cc] = v;
            sq += v * v;
        }
    if (sq != 0.0) node_nz[an] = 1;
}

// ---------------------------------------------------------------------------
// full-pivot ACA (cooperative; R double-buffered; one barrier per step)
// ---------------------------------------------------------------------------
struct MaxIdx {
    double v;
    long long i;
};
__device__ __forceinline__ MaxIdx better(MaxIdx p, MaxIdx q) {
    if (q.v > p.v || (q.v == p.v && q.i < p.i)) return q;
    return p;
}
__device__ __forceinline__ MaxIdx warp_best(MaxIdx m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        MaxIdx q;
        q.v = __shfl_xor_sync(0xffffffffu, m.v, o);
        q.i = __shfl_xor_sync(0xffffffffu, m.i, o);
        m = better(m, q);
    }
    return m;
}

// Full-pivot ACA over the whole grid (couplings too large for the cluster
// kernel).  Each CTA owns a strip of whole columns of R (all m rows, a
// multiple of 32 columns): per rank step it forms v = R[i, strip] / pivot once
// per column and u = R[:, j] once per row in shared memory, then updates its
// strip (R - u v, no FMA, as numpy's R - outer(u, v)) with coalesced row
// segments while it tracks the sum of squares and the row-major first
// largest |R|; one grid barrier per step.
__global__ void __launch_bounds__(256) aca_kernel(AcaParams p) {
    __shared__ double s_sum[8];
    __shared__ MaxIdx s_max[8];
    __shared__ double s_bc[4];
    __shared__ long long s_bi;
    extern __shared__ double s_uv[];        // u (m rows) then v (strip columns)
    const int m = p.m, nc = p.nc;
    const long long total = (long long)m * nc;
    const unsigned G = gridDim.x;
    const int strip = p.strip;                          // columns per CTA (a multiple of 32)
    double* s_u = s_uv;
    double* s_v = s_uv + m;
    const int c0 = min(nc, (int)blockIdx.x * strip), c1 = min(nc, c0 + strip);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int lane = tx, warp = ty;
    double* R[2] = {p.R0, p.R1};
    int cur = 0;

    auto reduce_local = [&](double lsum, MaxIdx lm) {
        lsum = wsum(lsum);
        lm = warp_best(lm);
        if (lane == 0) { s_sum[warp] = lsum; s_max[warp] = lm; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            MaxIdx b{-1.0, (long long)total};
            for (int w = 0; w < 8; ++w) { s += s_sum[w]; b = better(b, s_max[w]); }
            p.psum[blockIdx.x] = s;
            p.pmax[blockIdx.x] = b.v;
            p.pidx[blockIdx.x] = b.i;
        }
        __syncthreads();
    };
    // pass 0 over E
    {
        double ls = 0.0;
        MaxIdx lm{-1.0, (long long)total};
        for (int r = ty; r < m; r += 8)
            for (int c = c0 + tx; c < c1; c += 32) {
                const long long f = (long long)r * nc + c;
                const double v = R[0][f];
                ls += v * v;
                lm = better(lm, MaxIdx{fabs(v), f});
            }
        reduce_local(ls, lm);
    }
    int epoch = 0;
    if (!grid_sync(p.bar, G, p.spin_limit, epoch++)) return;
    double scale = 0.0, residual = 0.0;
    int k = 0;
    for (;; ++k) {
        // global reduction, same order in every CTA (warp 0, lanes stride the partials)
        if (warp == 0) {
            double s = 0.0;
            MaxIdx b{-1.0, (long long)total};
            for (unsigned c = lane; c < G; c += 32) {
                s += p.psum[c];
                b = better(b, MaxIdx{p.pmax[c], p.pidx[c]});
            }
            s = wsum(s);
            b = warp_best(b);
            if (lane == 0) { s_bc[0] = s; s_bc[1] = b.v; s_bi = b.i; }
        }
        __syncthreads();
        const double gsum = s_bc[0];
        const long long gi = s_bi;
        if (k == 0) {
            scale = sqrt(gsum);
            residual = scale > 0 ? 1.0 : 0.0;
        } else {
            residual = sqrt(gsum) / scale;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) p.hist[k] = residual;
        if (!(residual > p.rtol) || k >= p.cap) break;
        const int i = (int)(gi / nc), j = (int)(gi - (long long)i * nc);
        const double* Rc = R[cur];
        double* Rn = R[cur ^ 1];
        const double pivot = Rc[gi];
        if (!(fabs(pivot) > DBL_EPSILON * fmax(scale, DBL_MIN))) break;
        for (int r = threadIdx.x; r < m; r += blockDim.x) {
            const double u = Rc[(size_t)r * nc + j];
            s_u[r] = u;
            if (blockIdx.x == 0) p.U[(size_t)k * m + r] = u;
        }
        for (int c = c0 + (int)threadIdx.x; c < c1; c += blockDim.x) {
            const double v = Rc[(size_t)i * nc + c] / pivot;
            s_v[c - c0] = v;
            p.V[(size_t)k * nc + c] = v;
        }
        __syncthreads();
        double ls = 0.0;
        MaxIdx lm{-1.0, (long long)total};
        for (int r = ty; r < m; r += 8) {
            const double u = s_u[r];
            for (int c = c0 + tx; c < c1; c += 32) {
                const long long f = (long long)r * nc + c;
                const double val = __dsub_rn(Rc[f], __dmul_rn(u, s_v[c - c0]));  // numpy: R - outer(u, v), no FMA
                Rn[f] = val;
                ls += val * val;
                lm = better(lm, MaxIdx{fabs(val), f});
            }
        }
        reduce_local(ls, lm);
        cur ^= 1;
        if (!grid_sync(p.bar, G, p.spin_limit, epoch++)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *p.rank = k;
        *p.err = residual;
    }
}

// ---------------------------------------------------------------------------
// small dense FP64 algebra
// ---------------------------------------------------------------------------
// C = alpha op(A) op(B) + beta C (row-major; op = transpose when t* != 0) in FP64 on the tensor cores (mma.sync m8n8k4, .f64: d = a b + c
// per 8 x 8 x 4 step).  A CTA of four warps takes a 32 x 32 tile of C, the K loop in steps of 32
// through shared memory; warp w owns rows 8 w .. 8 w + 7 of the tile as four 8 x 8 accumulator
// tiles that share its A fragment.  Fragments (PTX m8n8k4 .f64): lane l holds A(l / 4, l % 4),
// B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + i), i < 2.  The sizes may come from the device (rank).
__global__ void __launch_bounds__(128) gemm_kernel(GemmArgs g) {
    __shared__ double As[32][33];   // [row][k]
    __shared__ double Bs[32][33];   // [k][col]
    const int M = g.dM ? *g.dM : g.M, N = g.dN ? *g.dN : g.N, K = g.dK ? *g.dK : g.K;
    const int bm = blockIdx.y * 32, bn = blockIdx.x * 32;
    if (bm >= M || bn >= N) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gr = lane >> 2, gc = lane & 3;
    double acc[4][2] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    for (int k0 = 0; k0 < K; k0 += 32) {
        for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
            const int rr = e >> 5, cc = e & 31;
            const int row = bm + rr, kk = k0 + cc;
            double va = 0.0;
            if (row < M && kk < K) va = g.tA ? g.A[(size_t)kk * g.lda + row] : g.A[(size_t)row * g.lda + kk];
            As[rr][cc] = va;
            const int kr = k0 + rr, col = bn + cc;
            double vb = 0.0;
            if (kr < K && col < N) vb = g.tB ? g.B[(size_t)col * g.ldb + kr] : g.B[(size_t)kr * g.ldb + col];
            Bs[rr][cc] = vb;
        }
        __syncthreads();
#pragma unroll
        for (int k4 = 0; k4 < 8; ++k4) {
            const double av = As[8 * warp + gr][4 * k4 + gc];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const double bv = Bs[4 * k4 + gc][8 * t + gr];
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                             : "+d"(acc[t][0]), "+d"(acc[t][1])
                             : "d"(av), "d"(bv));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int row = bm + 8 * warp + gr, col = bn + 8 * t + 2 * gc + i;
            if (row < M && col < N) {
                double* c = g.C + (size_t)row * g.ldc + col;
                const double prev = g.beta == 0.0 ? 0.0 : g.beta * *c;
                *c = g.alpha * acc[t][i] + prev;
            }
        }
}

// Cholesky A = L L^T (lower, row-major) in one CTA; L overwrites Lout.
// Shared memory holds the matrix when it fits, else it works in Lout.
__global__ void __launch_bounds__(1024) cholesky_kernel(const double* A, int m, double* Lout, int use_smem,
                                                        int* bad) {
    extern __shared__ double sm[];
    double* L = use_smem ? sm : Lout;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) L[e] = A[e];
    __syncthreads();
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    for (int j = 0; j < m; ++j) {
        if (threadIdx.x == 0) {
            const double d = L[(size_t)j * m + j];
            if (!(d > 0.0) || !isfinite(d)) { s_bad = 1; L[(size_t)j * m + j] = 1.0; }
            else L[(size_t)j * m + j] = sqrt(d);
        }
        __syncthreads();
        const double dj = L[(size_t)j * m + j];
        for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) L[(size_t)i * m + j] /= dj;
        __syncthreads();
        const int rem = m - j - 1;
        for (int e = threadIdx.x; e < rem * rem; e += blockDim.x) {
            const int i = j + 1 + e / rem, l = j + 1 + e % rem;
            if (l <= i) L[(size_t)i * m + l] -= L[(size_t)i * m + j] * L[(size_t)l * m + j];
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int i = e / m, l = e % m;
        Lout[e] = l <= i ? L[e] : 0.0;
    }
    if (threadIdx.x == 0 && s_bad) atomicAdd(bad, 1);
}

// X = A^-1 B with A = L L^T; B, X row-major m x ncol (may alias).  One warp
// per right-hand-side column: forward then backward substitution.
__global__ void chol_solve_kernel(const double* L, int m, const double* B, int ldb, double* X, int ldx,
                                  int ncol, const int* dncol, double* work) {
    const int nc = dncol ? *dncol : ncol;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= nc) return;
    double* y = work + (size_t)gw * m;
    for (int i = 0; i < m; ++i) {
        double s = 0.0;
        for (int k = lane; k < i; k += 32) s += L[(size_t)i * m + k] * y[k];
        s = wsum(s);
        if (lane == 0) y[i] = (B[(size_t)i * ldb + gw] - s) / L[(size_t)i * m + i];
        __syncwarp();
    }
    for (int i = m - 1; i >= 0; --i) {
        double s = 0.0;
        for (int k = i + 1 + lane; k < m; k += 32) s += L[(size_t)k * m + i] * y[k];
        s = wsum(s);
        if (lane == 0) y[i] = (y[i] - s) / L[(size_t)i * m + i];
        __syncwarp();
    }
    for (int i = lane; i < m; i += 32) X[(size_t)i * ldx + gw] = y[i];
}

// P = A^-1 for an SPD A in one 1024-thread CTA by in-place Gauss-Jordan
// elimination without pivoting (for SPD A its pivots are the squared Cholesky
// diagonal, so a pivot <= 0 flags a non-SPD block exactly as LLT does).  Each
// of the m steps stages row and column k, then updates all m^2 entries in
// parallel with one reciprocal: two barriers per step, no long dependent chain.
__global__ void __launch_bounds__(1024) gj_inverse_kernel(const double* A, int m, double* P, int* bad) {
    extern __shared__ double W[];
    const int ld = m + 1;
    double* rowk = W + (size_t)m * ld;
    double* colk = rowk + m;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int i = ty; i < m; i += 32)
        for (int j = tx; j < m; j += 32) W[i * ld + j] = A[(size_t)i * m + j];
    __syncthreads();
    bool ok = true;
    for (int k = 0; k < m; ++k) {
        double p = W[k * ld + k];
        if (!(p > 0.0) || !isfinite(p)) { ok = false; p = 1.0; }
        const double rp = 1.0 / p;
        for (int t = threadIdx.x; t < m; t += 1024) {
            rowk[t] = W[k * ld + t];
            colk[t] = W[t * ld + k];
        }
        __syncthreads();
        for (int i = ty; i < m; i += 32) {
            const double ci = colk[i];
            for (int j = tx; j < m; j += 32) {
                double v;
                if (i == k) v = (j == k) ? rp : rowk[j] * rp;
                else if (j == k) v = -ci * rp;
                else v = W[i * ld + j] - ci * rowk[j] * rp;
                W[i * ld + j] = v;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && !ok) atomicAdd(bad, 1);
    for (int i = ty; i < m; i += 32)
        for (int j = tx; j < m; j += 32) P[(size_t)i * m + j] = W[i * ld + j];
}

// The same elimination for m <= 144 with the matrix held in registers: thread
// (ty, tx) of a 16 x 32 grid owns rows ty + 16 r (r < 9) and columns tx + 32 c
// (c < 5) for the whole inversion.  Step k: the owners of row k and column k
// publish them (and the reciprocal pivot) in shared memory, one barrier, then
// every thread updates its own entries.  The published row and column alternate
// between two buffers, so one barrier per step keeps the next step's writers off
// this step's readers.  Per step a thread reads 14 shared values instead of
// streaming the whole matrix through shared memory.
constexpr int kGjR = 9, kGjC = 5, kGjMax = 16 * kGjR;
constexpr int kGbR = 3, kGbMax = 32 * kGbR;  // the 1024-thread kernel below
__global__ void __launch_bounds__(512) gj_inverse_reg_kernel(const double* A, int ld, const int* dk, double* P, int* bad) {
    __shared__ double s_row[2][32 * kGjC], s_col[2][kGjMax], s_rp[2];
    __shared__ int s_bad;
    int m = ld;
    if (dk) {  // the leading *dk x *dk block of an ld x ld matrix; ranks the 1024-thread kernel took are skipped
        const int kd = *dk;
        if (kd <= kGbMax) return;
        m = min(ld, kd);
    }
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double w[kGjR][kGjC];
#pragma unroll
    for (int r = 0; r < kGjR; ++r)
#pragma unroll
        for (int c = 0; c < kGjC; ++c) {
            const int i = ty + 16 * r, j = tx + 32 * c;
            w[r][c] = (i < m && j < m) ? A[(size_t)i * ld + j] : 0.0;
        }
    if (threadIdx.x == 0) s_bad = 0;
    for (int k = 0; k < m; ++k) {
        const int b = k & 1, kr = k >> 4, kc = k >> 5;
        if (ty == (k & 15)) {
#pragma unroll
            for (int r = 0; r < kGjR; ++r)
                if (r == kr)
#pragma unroll
                    for (int c = 0; c < kGjC; ++c) {
                        const int j = tx + 32 * c;
                        if (j < m) s_row[b][j] = w[r][c];
                    }
        }
        if (tx == (k & 31)) {
#pragma unroll
            for (int c = 0; c < kGjC; ++c)
                if (c == kc)
#pragma unroll
                    for (int r = 0; r < kGjR; ++r) {
                        const int i = ty + 16 * r;
                        if (i < m) s_col[b][i] = w[r][c];
                        if (i == k) {
                            double p = w[r][c];
                            if (!(p > 0.0) || !isfinite(p)) { s_bad = 1; p = 1.0; }
                            s_rp[b] = 1.0 / p;
                        }
                    }
        }
        __syncthreads();
        const double rp = s_rp[b];
        double rs[kGjC];
#pragma unroll
        for (int c = 0; c < kGjC; ++c) {
            const int j = tx + 32 * c;
            rs[c] = j < m ? s_row[b][j] * rp : 0.0;  // pivot row / pivot
        }
        // every entry: w_ij - c_i (row_j / p); then the owners of column k and row k overwrite
        // theirs (-c_i / p, row_j / p, 1 / p) -- a warp-uniform branch for the row, one lane for the column
#pragma unroll
        for (int r = 0; r < kGjR; ++r) {
            const int i = ty + 16 * r;
            const double ci = i < m ? s_col[b][i] : 0.0;
#pragma unroll
            for (int c = 0; c < kGjC; ++c) w[r][c] = fma(-ci, rs[c], w[r][c]);
        }
        if (tx == (k & 31)) {
#pragma unroll
            for (int c = 0; c < kGjC; ++c)
                if (c == kc)
#pragma unroll
                    for (int r = 0; r < kGjR; ++r) {
                        const int i = ty + 16 * r;
                        w[r][c] = i < m ? -s_col[b][i] * rp : 0.0;
                    }
        }
        if (ty == (k & 15)) {
#pragma unroll
            for (int r = 0; r < kGjR; ++r)
                if (r == kr)
#pragma unroll
                    for (int c = 0; c < kGjC; ++c) w[r][c] = (tx + 32 * c == k) ? rp : rs[c];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) atomicAdd(bad, 1);
#pragma unroll
    for (int r = 0; r < kGjR; ++r)
#pragma unroll
        for (int c = 0; c < kGjC; ++c) {
            const int i = ty + 16 * r, j = tx + 32 * c;
            if (i < m && j < m) P[(size_t)i * ld + j] = w[r][c];
        }
}

// The same elimination for blocks of at most 96 rows, one 1024-thread CTA per block: thread
// (ty, tx) of a 32 x 32 grid owns rows ty + 32 r and columns tx + 32 c (r, c < 3), nine entries.
// A warp holds whole rows, so the pivot column's entries of its rows come by shuffle from lane
// k mod 32; only the pivot row (one warp) and the reciprocal pivot (one lane) go through shared
// memory, double-buffered, one barrier per step.  A block is the set of rows and columns
// idx[ptr[g] .. ptr[g + 1]) of the m x m matrix (idx null: the whole matrix, one block; dk
// non-null: the leading *dk x *dk block).  Gauss-Jordan without pivoting never mixes two blocks
// of a block-diagonal matrix (the products across them are exact zeros), so inverting the blocks
// apart gives the whole inverse bit for bit; entries of P outside the blocks are left to the caller.
__device__ __forceinline__ double sel3(const double (&v)[3], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]); }

__global__ void __launch_bounds__(1024) gj_inverse_blocks_kernel(const double* A, int m, const int* ptr, const int* idx,
                                                                 const int* dk, double* P, int* bad) {
    __shared__ double s_row[2][kGbMax], s_rp[2];
    __shared__ int s_bad;
    const int g = blockIdx.x;
    const int b0 = ptr ? ptr[g] : 0;
    int mb = ptr ? ptr[g + 1] - b0 : m;
    if (dk) {  // the leading *dk x *dk block (no ptr); larger ranks go to the 512-thread kernel
        const int kd = *dk;
        if (kd > kGbMax) return;
        mb = min(mb, kd);
    }
    const int* ix = idx ? idx + b0 : nullptr;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    int gi[kGbR], gj[kGbR];
#pragma unroll
    for (int r = 0; r < kGbR; ++r) {
        const int i = ty + 32 * r, j = tx + 32 * r;
        gi[r] = i < mb ? (ix ? ix[i] : i) : 0;
        gj[r] = j < mb ? (ix ? ix[j] : j) : 0;
    }
    double w[kGbR][kGbR];
#pragma unroll
    for (int r = 0; r < kGbR; ++r)
#pragma unroll
        for (int c = 0; c < kGbR; ++c) {
            const int i = ty + 32 * r, j = tx + 32 * c;
            w[r][c] = (i < mb && j < mb) ? A[(size_t)gi[r] * m + gj[c]] : 0.0;
        }
    if (threadIdx.x == 0) s_bad = 0;
    // the 32-step blocks unrolled: the pivot's register (entry kk of a thread's rows and columns)
    // is a compile-time index, so no run-time select sits on a step's path
#pragma unroll
    for (int kk = 0; kk < kGbR; ++kk) {
        for (int ko = 0; ko < 32; ++ko) {
            const int k = 32 * kk + ko;
            if (k >= mb) break;  // uniform
            const int b = k & 1;
            double ci[kGbR];
#pragma unroll
            for (int r = 0; r < kGbR; ++r) ci[r] = __shfl_sync(0xffffffffu, w[r][kk], ko);  // column k
            if (ty == ko) {  // the pivot row's warp publishes it, its pivot lane the reciprocal
#pragma unroll
                for (int c = 0; c < kGbR; ++c) s_row[b][tx + 32 * c] = w[kk][c];
                if (tx == ko) {
                    double pv = ci[kk];
                    if (!(pv > 0.0) || !isfinite(pv)) { s_bad = 1; pv = 1.0; }
                    s_rp[b] = 1.0 / pv;
                }
            }
            __syncthreads();
            const double rp = s_rp[b];
            double rs[kGbR];
#pragma unroll
            for (int c = 0; c < kGbR; ++c) rs[c] = s_row[b][tx + 32 * c] * rp;  // pivot row / pivot
#pragma unroll
            for (int r = 0; r < kGbR; ++r)
#pragma unroll
                for (int c = 0; c < kGbR; ++c) w[r][c] = fma(-ci[r], rs[c], w[r][c]);
            // the owners of column k and row k overwrite theirs: -c_i / p, row_j / p, 1 / p
            if (tx == ko) {
#pragma unroll
                for (int r = 0; r < kGbR; ++r) w[r][kk] = -ci[r] * rp;
            }
            if (ty == ko) {
#pragma unroll
                for (int c = 0; c < kGbR; ++c) w[kk][c] = (tx + 32 * c == k) ? rp : rs[c];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_bad) atomicAdd(bad, 1);
#pragma unroll
    for (int r = 0; r < kGbR; ++r)
#pragma unroll
        for (int c = 0; c < kGbR; ++c) {
            const int i = ty + 32 * r, j = tx + 32 * c;
            if (i < mb && j < mb) P[(size_t)gi[r] * m + gj[c]] = w[r][c];
        }
}

// C (k x k, row-major, k from device, k <= 96) = L diag(d) L^T in one 1024-thread CTA, the
// matrix in registers as in the kernel above (thread (ty, tx): rows ty + 32 r, columns tx + 32 c).
// Step j: a warp takes column j of its rows by shuffle and publishes it, one barrier, then every
// entry below and right of (j, j) takes W_il -= (W_ij / d_j) W_lj, the operations and order of
// the shared-memory kernel below; only the lower triangle is read.  Returns at once when k > 96.
__global__ void __launch_bounds__(1024) ldlt_reg_kernel(const double* C, int kmax, const int* dk, double* L, double* d,
                                                        int* bad) {
    __shared__ double s_col[2][kGbMax], s_rd[2];
    __shared__ int s_bad;
    const int k = *dk;
    if (k > kGbMax) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double w[kGbR][kGbR];
#pragma unroll
    for (int r = 0; r < kGbR; ++r)
#pragma unroll
        for (int c = 0; c < kGbR; ++c) {
            const int i = ty + 32 * r, l = tx + 32 * c;
            w[r][c] = (i < k && l < k && l <= i) ? 0.5 * (C[(size_t)i * kmax + l] + C[(size_t)l * kmax + i]) : 0.0;
        }
    if (threadIdx.x == 0) s_bad = 0;
    // the 32-step blocks unrolled: the pivot column's register is a compile-time index
#pragma unroll
    for (int jj = 0; jj < kGbR; ++jj) {
        for (int jo = 0; jo < 32; ++jo) {
            const int j = 32 * jj + jo;
            if (j >= k) break;  // uniform
            const int b = j & 1;
            double ci[kGbR];
#pragma unroll
            for (int r = 0; r < kGbR; ++r) ci[r] = __shfl_sync(0xffffffffu, w[r][jj], jo);  // W[i][j]
            if (tx < kGbR) s_col[b][ty + 32 * tx] = sel3(ci, tx);
            if (ty == jo && tx == jo) {
                const double dj = ci[jj];
                const bool okj = isfinite(dj) && dj != 0.0;
                if (!okj) s_bad = 1;
                s_rd[b] = 1.0 / (okj ? dj : 1.0);
            }
            __syncthreads();
            const double rd = s_rd[b];
            double cl[kGbR];
#pragma unroll
            for (int c = 0; c < kGbR; ++c) cl[c] = (tx + 32 * c > j) ? s_col[b][tx + 32 * c] : 0.0;
#pragma unroll
            for (int r = 0; r < kGbR; ++r) {
                const double wij = (ty + 32 * r > j) ? ci[r] * rd : 0.0;
#pragma unroll
                for (int c = 0; c < kGbR; ++c) w[r][c] = fma(-wij, cl[c], w[r][c]);
            }
            if (tx == jo) {  // column j becomes L[:, j] below the diagonal
#pragma unroll
                for (int r = 0; r < kGbR; ++r)
                    if (ty + 32 * r > j) w[r][jj] = ci[r] * rd;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kGbR; ++r)
#pragma unroll
        for (int c = 0; c < kGbR; ++c) {
            const int i = ty + 32 * r, l = tx + 32 * c;
            if (i < kmax && l < kmax) {
                double v = 0.0;
                if (i < k && l < k) v = (l < i) ? w[r][c] : (l == i ? 1.0 : 0.0);
                L[(size_t)i * kmax + l] = v;
                if (i == l) d[i] = i < k ? w[r][c] : 0.0;
            }
        }
    for (int e = threadIdx.x; e < kmax * kmax; e += blockDim.x) {  // beyond the register tiles (kmax > 96)
        const int i = e / kmax, l = e - i * kmax;
        if (i >= kGbMax || l >= kGbMax) L[e] = 0.0;
    }
    for (int i = kGbMax + threadIdx.x; i < kmax; i += blockDim.x) d[i] = 0.0;
    if (threadIdx.x == 0 && s_bad) atomicAdd(bad, 1);
}

// P = A^-1 for an SPD A (m <= 160) in one 1024-thread CTA: Cholesky in
// shared memory (2-D trailing update, two barriers per column), then each warp
// solves L L^T x = e_c for its columns with the vector held in registers
// (lane l owns entries l, l+32, ...).
constexpr int kCholQ = 5;  // 32 * 5 = 160 rows in registers
__global__ void __launch_bounds__(1024) chol_inverse_kernel(const double* A, int m, double* P, int* bad) {
    extern __shared__ double L[];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int ld = m + 1;  // odd row stride: column walks hit distinct banks
    for (int e = threadIdx.x; e < m * m; e += 1024) L[(e / m) * ld + e % m] = A[e];
    __syncthreads();
    bool ok = true;
    for (int j = 0; j < m; ++j) {
        double d = L[j * ld + j];
        if (!(d > 0.0) || !isfinite(d)) { ok = false; d = 1.0; }
        const double dj = sqrt(d);
        __syncthreads();
        if (threadIdx.x == 0) L[j * ld + j] = dj;
        for (int i = j + 1 + threadIdx.x; i < m; i += 1024) L[i * ld + j] /= dj;
        __syncthreads();
        for (int i = j + 1 + ty; i < m; i += 32) {
            const double lij = L[i * ld + j];
            for (int l = j + 1 + tx; l <= i; l += 32)
                if (HSC_IN(i * ld + l < m * ld && l * ld + j < m * ld, 300, i * ld + l)) L[i * ld + l] -= lij * L[l * ld + j];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && !ok) atomicAdd(bad, 1);
    // columns of the inverse
    for (int c = ty; c < m; c += 32) {
        double y[kCholQ];
#pragma unroll
        for (int q = 0; q < kCholQ; ++q) y[q] = 0.0;
        for (int i = 0; i < m; ++i) {                       // L y = e_c
            double sacc = 0.0;
#pragma unroll
            for (int q = 0; q < kCholQ; ++q) {
                const int k = 32 * q + tx;
                if (k < i) sacc += L[i * ld + k] * y[q];
            }
            sacc = wsum(sacc);
            const double v = ((i == c ? 1.0 : 0.0) - sacc) / L[i * ld + i];
#pragma unroll
            for (int q = 0; q < kCholQ; ++q)
                if (32 * q + tx == i) y[q] = v;
        }
        for (int i = m - 1; i >= 0; --i) {                  // L^T x = y
            double sacc = 0.0;
#pragma unroll
            for (int q = 0; q < kCholQ; ++q) {
                const int k = 32 * q + tx;
                if (k > i && k < m) sacc += L[k * ld + i] * y[q];
            }
            sacc = wsum(sacc);
#pragma unroll
            for (int q = 0; q < kCholQ; ++q)
                if (32 * q + tx == i) y[q] = (y[q] - sacc) / L[i * ld + i];
        }
#pragma unroll
        for (int q = 0; q < kCholQ; ++q) {
            const int i = 32 * q + tx;
            if (i < m && HSC_IN(c < m, 301, c)) P[(size_t)i * m + c] = y[q];
        }
    }
}

// C (k x k, row-major, k from device) = L diag(d) L^T in one CTA: L unit lower
// (row-major, ld kmax) and d written out; C symmetrised first.
__global__ void __launch_bounds__(1024) ldlt_kernel(double* C, int kmax, const int* dk, double* L, double* d,
                                                    int use_smem, int* bad) {
    extern __shared__ double sm[];
    const int k = *dk;
    if (k <= kGbMax) return;  // the register kernel took it
    double* W = use_smem ? sm : C;
    const int ldw = use_smem ? k + 1 : kmax;  // odd stride in shared memory
    for (int e = threadIdx.x; e < k * k; e += blockDim.x) {  // lower triangle only (in place when W == C)
        const int i = e / k, l = e % k;
        if (l <= i) W[(size_t)i * ldw + l] = 0.5 * (C[(size_t)i * kmax + l] + C[(size_t)l * kmax + i]);
    }
    __syncthreads();
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    __shared__ double colj[kMaxRank];
    for (int j = 0; j < k; ++j) {
        const double dj = W[(size_t)j * ldw + j];
        const bool okj = isfinite(dj) && dj != 0.0;
        if (threadIdx.x == 0 && !okj) s_bad = 1;
        const double rd = 1.0 / (okj ? dj : 1.0);
        for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) colj[i] = W[(size_t)i * ldw + j];
        __syncthreads();
        // trailing update with the unscaled column j, then store L[:, j]
        for (int i = j + 1 + ty; i < k; i += 32) {
            const double wij = colj[i] * rd;
            for (int l = j + 1 + tx; l <= i; l += 32) W[(size_t)i * ldw + l] -= wij * colj[l];
        }
        for (int i = j + 1 + threadIdx.x; i < k; i += blockDim.x) W[(size_t)i * ldw + j] = colj[i] * rd;
        __syncthreads();
    }
    for (int e = threadIdx.x; e < kmax * kmax; e += blockDim.x) {
        const int i = e / kmax, l = e % kmax;
        double v = 0.0;
        if (i < k && l < k) v = (l < i) ? W[(size_t)i * ldw + l] : (l == i ? 1.0 : 0.0);
        L[e] = v;
    }
    for (int j = threadIdx.x; j < kmax; j += blockDim.x) d[j] = j < k ? W[(size_t)j * ldw + j] : 0.0;
    if (threadIdx.x == 0 && s_bad) atomicAdd(bad, 1);
}

// 12x12 diagonal-block Cholesky inverses (one thread per body) into a dense
// qm x qm block-diagonal Binv (row-major)
__global__ void block12_inverse_kernel(const double* A, int qm, double* Binv, int* bad) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= qm / 12) return;
    double L[12][12];
    const int o = 12 * b;
    for (int i = 0; i < 12; ++i)
        for (int j = 0; j < 12; ++j) L[i][j] = A[(size_t)(o + i) * qm + o + j];
    bool ok = true;
    for (int j = 0; j < 12; ++j) {
        double d = L[j][j];
        for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
        if (!(d > 0.0) || !isfinite(d)) { ok = false; d = 1.0; }
        d = sqrt(d);
        L[j][j] = d;
        for (int i = j + 1; i < 12; ++i) {
            double s = L[i][j];
            for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
            L[i][j] = s / d;
        }
    }
    if (!ok) atomicAdd(bad, 1);
    for (int c = 0; c < 12; ++c) {
        double y[12];
        for (int i = 0; i < 12; ++i) {
            double s = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
            y[i] = s / L[i][i];
        }
        for (int i = 11; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < 12; ++k) s -= L[k][i] * y[k];
            y[i] = s / L[i][i];
        }
        for (int i = 0; i < 12; ++i) Binv[(size_t)(o + i) * qm + o + c] = y[i];
    }
}

__global__ void axpby_mat_kernel(double* Y, const double* X, double a, double b, int n, int diag_m, double diag_add) {
    // Y = a X + b Y (+ diag_add on the diagonal of an m x m matrix when diag_m > 0)
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    double v = a * (X ? X[e] : 0.0) + b * Y[e];
    if (diag_m > 0 && (e / diag_m) == (e % diag_m)) v += diag_add;
    Y[e] = v;
}

__global__ void symmetrize_kernel(double* P, int m) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m * m) return;
    const int i = e / m, j = e % m;
    if (j <= i) return;
    const double v = 0.5 * (P[(size_t)i * m + j] + P[(size_t)j * m + i]);
    P[(size_t)i * m + j] = v;
    P[(size_t)j * m + i] = v;
}

__global__ void frob_kernel(const double* X, int n, double* out) {
    double s = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) s += X[e] * X[e];
    s = bsum(s);
    if (threadIdx.x == 0) *out = s;
}

// ---------------------------------------------------------------------------
// vectors
// ---------------------------------------------------------------------------
// split b (contiguous N) into bq (qm) and node-padded FEM part bf; internal node i
// is the caller's node perm[i] (perm null: the identity)
__global__ void split_rhs_kernel(const double* b, int qo, int qm, int fo, int n, const int* perm, double* bq,
                                 double* bf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < qm) bq[i] = b[qo + i];
    if (i < n) {
        const double* s = b + fo + 3 * (size_t)(perm ? perm[i] : i);
        bf[4 * (size_t)i] = s[0];
        bf[4 * (size_t)i + 1] = s[1];
        bf[4 * (size_t)i + 2] = s[2];
        bf[4 * (size_t)i + 3] = 0.0;
    }
}

// c = W^T bq (k from device); one warp per output
__global__ void wt_vec_kernel(const double* W, int qm, int kmax, const int* dk, const double* bq, double* c) {
    const int k = *dk;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= k) return;
    double s = 0.0;
    for (int i = lane; i < qm; i += 32) s += W[(size_t)i * kmax + gw] * bq[i];
    s = wsum(s);
    if (lane == 0) c[gw] = s;
}

// sum_{j < n} M[j a + i] v[j] for the CTA's 32 consecutive i (lane of warp 0 on return; other
// threads return 0): the 8 warps take j = g, g + 8, ... (coalesced over i, four loads in flight
// per thread), then warp 0 adds the 8 group sums in group order (deterministic)
constexpr int kColGroups = 8;
__device__ __forceinline__ double col_sums_32x8(const double* M, int a, int n, const double* v, int i) {
    __shared__ double s_part[kColGroups][32];
    const int lane = threadIdx.x & 31, g = threadIdx.x >> 5;
    double s0 = 0.0, s1 = 0.0;
    if (i < a) {
        int j = g;
        for (; j + kColGroups < n; j += 2 * kColGroups) {
            s0 += M[(size_t)j * a + i] * v[j];
            s1 += M[(size_t)(j + kColGroups) * a + i] * v[j + kColGroups];
        }
        if (j < n) s0 += M[(size_t)j * a + i] * v[j];
    }
    s_part[g][lane] = s0 + s1;
    __syncthreads();
    double t = 0.0;
    if (g == 0)
        for (int h = 0; h < kColGroups; ++h) t += s_part[h][lane];
    return t;
}

// rhs[act_i] -= (V c)_i ; V column-major a x kmax; 32 coupled dofs per 256-thread CTA
__global__ void __launch_bounds__(32 * kColGroups) rhs_lowrank_kernel(const double* V, int a, const int* dk,
                                                                      const double* c, const int* act, double* rhs) {
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const double s = col_sums_32x8(V, a, *dk, c, i);
    if (threadIdx.x < 32 && i < a) {
        const int dof = act[i];
        rhs[4 * (size_t)(dof / 3) + dof % 3] -= s;
    }
}

// t = V^T x[act] ; a 256-thread CTA per column, its threads over the coupled dofs (every load
// in flight at once), then a fixed-order CTA reduction
__global__ void __launch_bounds__(256) vt_x_kernel(const double* V, int a, const int* dk, const int* act,
                                                   const double* x, double* t) {
    __shared__ double s_w[8];
    const int j = blockIdx.x;
    if (j >= *dk) return;  // uniform in the CTA
    const double* vj = V + (size_t)j * a;
    double s0 = 0.0, s1 = 0.0;
    int i = threadIdx.x;
    for (; i + 256 < a; i += 512) {
        const int d0 = act[i], d1 = act[i + 256];
        s0 += vj[i] * x[4 * (size_t)(d0 / 3) + d0 % 3];
        s1 += vj[i + 256] * x[4 * (size_t)(d1 / 3) + d1 % 3];
    }
    if (i < a) {
        const int d0 = act[i];
        s0 += vj[i] * x[4 * (size_t)(d0 / 3) + d0 % 3];
    }
    const double s = wsum(s0 + s1);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < 8; ++w) r += s_w[w];
        t[j] = r;
    }
}

// dq = P bq - W t  (one warp per ABD row), written to x_out[qo + i]
__global__ void backsub_kernel(const double* P, const double* W, int qm, int kmax, const int* dk,
                               const double* bq, const double* t, double* xq_out, double* xq_copy) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= qm) return;
    const int k = *dk;
    double s = 0.0;
    for (int j = lane; j < qm; j += 32) s += P[(size_t)gw * qm + j] * bq[j];
    for (int j = lane; j < k; j += 32) s -= W[(size_t)gw * kmax + j] * t[j];
    s = wsum(s);
    if (lane == 0) {
        xq_out[gw] = s;
        if (xq_copy) xq_copy[gw] = s;
    }
}

__global__ void scatter_x_kernel(const double* xpad, int n, int fo, const int* perm, double* xout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double* d = xout + fo + 3 * (size_t)(perm ? perm[i] : i);
    d[0] = xpad[4 * (size_t)i];
    d[1] = xpad[4 * (size_t)i + 1];
    d[2] = xpad[4 * (size_t)i + 2];
}

__global__ void gather_x_kernel(const double* x, int n, int fo, const int* perm, double* xpad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* s = x + fo + 3 * (size_t)(perm ? perm[i] : i);
    xpad[4 * (size_t)i] = s[0];
    xpad[4 * (size_t)i + 1] = s[1];
    xpad[4 * (size_t)i + 2] = s[2];
    xpad[4 * (size_t)i + 3] = 0.0;
}

// y_f = D x_f (FP64, row-owner) for the node-padded x; written contiguously
// into y_out[fo + 3 i] (y_out may be null) and node-padded into ypad
__global__ void bsr_spmv64_kernel(const int* rowptr, const int* colidx, const double* v64, int nnz, int n,
                                  const double* xpad, double* ypad) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = tid >> 2, sub = tid & 3;
    double a0 = 0, a1 = 0, a2 = 0;
    if (row < n) {
        for (int k = rowptr[row] + sub; k < rowptr[row + 1]; k += 4) {
            const int c = colidx[k];
            const double x0 = xpad[4 * (size_t)c], x1 = xpad[4 * (size_t)c + 1], x2 = xpad[4 * (size_t)c + 2];
            const double* v = v64 + k;
            a0 += v[0] * x0 + v[(size_t)nnz] * x1 + v[2 * (size_t)nnz] * x2;
            a1 += v[3 * (size_t)nnz] * x0 + v[4 * (size_t)nnz] * x1 + v[5 * (size_t)nnz] * x2;
            a2 += v[6 * (size_t)nnz] * x0 + v[7 * (size_t)nnz] * x1 + v[8 * (size_t)nnz] * x2;
        }
    }
#pragma unroll
    for (int o = 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (row < n && sub == 0) {
        ypad[4 * (size_t)row] = a0;
        ypad[4 * (size_t)row + 1] = a1;
        ypad[4 * (size_t)row + 2] = a2;
        ypad[4 * (size_t)row + 3] = 0.0;
    }
}

// The same product read straight from the caller's one-triangle BCOO through
// the row-owner plan (src = 2 t + transposed), for a single SpMV with fresh
// values: no refill of the BSR planes, each block read once per direction.
__global__ void bcoo_row_spmv_kernel(const int* rowptr, const int* colidx, const int* src, const double* values, int n,
                                     const double* xpad, double* ypad) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = tid >> 2, sub = tid & 3;
    double a0 = 0, a1 = 0, a2 = 0;
    if (row < n) {
        for (int k = rowptr[row] + sub; k < rowptr[row + 1]; k += 4) {
            const int c = colidx[k];
            const int packed = src[k];
            const double* B = values + 9 * (size_t)(packed >> 1);  // B(r, c) at r + 3 c
            const double x0 = xpad[4 * (size_t)c], x1 = xpad[4 * (size_t)c + 1], x2 = xpad[4 * (size_t)c + 2];
            double b[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) b[e] = B[e];
            if (packed & 1) {  // the mirrored block: B^T
                a0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
                a1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
                a2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
            } else {
                a0 += b[0] * x0 + b[3] * x1 + b[6] * x2;
                a1 += b[1] * x0 + b[4] * x1 + b[7] * x2;
                a2 += b[2] * x0 + b[5] * x1 + b[8] * x2;
            }
        }
    }
#pragma unroll
    for (int o = 2; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (row < n && sub == 0) {
        ypad[4 * (size_t)row] = a0;
        ypad[4 * (size_t)row + 1] = a1;
        ypad[4 * (size_t)row + 2] = a2;
        ypad[4 * (size_t)row + 3] = 0.0;
    }
}

// y_f[act_c] += sum_r E[r, c] xq[r]   (32 active columns per 256-thread CTA)
__global__ void __launch_bounds__(32 * kColGroups) et_xq_kernel(const double* E, int qm, int a, const int* act,
                                                                const double* xq, double* ypad) {
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const double s = col_sums_32x8(E, a, qm, xq, c);
    if (threadIdx.x < 32 && c < a) {
        const int dof = act[c];
        ypad[4 * (size_t)(dof / 3) + dof % 3] += s;
    }
}

// yq = A xq + E x_f[act] in two passes: one warp per (ABD row, chunk of
// kRowChunk coupled columns) writes a partial (chunk 0 also takes the A row),
// then one thread per row sums its partials in chunk order -- enough warps to
// stream a wide E (144 x 25,518 on the 1 M-tet torus), deterministic sums.
__global__ void abd_rows_part_kernel(const double* A, const double* E, int qm, int a, const int* act,
                                     const double* xq, const double* xpad, int nchunk, double* part) {
    const int r = blockIdx.y * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int chunk = blockIdx.x;
    if (r >= qm || chunk >= nchunk) return;
    double s = 0.0;
    if (chunk == 0)
        for (int j = lane; j < qm; j += 32) s += A[(size_t)r * qm + j] * xq[j];
    const int c1 = min(a, (chunk + 1) * kRowChunk);
    for (int c = chunk * kRowChunk + lane; c < c1; c += 32) {
        const int dof = act[c];
        s += E[(size_t)r * a + c] * xpad[4 * (size_t)(dof / 3) + dof % 3];
    }
    s = wsum(s);
    if (lane == 0) part[(size_t)r * nchunk + chunk] = s;
}

__global__ void abd_rows_sum_kernel(const double* part, int qm, int nchunk, double* yq) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= qm) return;
    double s = 0.0;
    for (int k = 0; k < nchunk; ++k) s += part[(size_t)r * nchunk + k];
    yq[r] = s;
}

// yq = A xq + E x_f[act]   (one warp per ABD row)
__global__ void abd_rows_kernel(const double* A, const double* E, int qm, int a, const int* act,
                                const double* xq, const double* xpad, double* yq) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= qm) return;
    double s = 0.0;
    for (int j = lane; j < qm; j += 32) s += A[(size_t)gw * qm + j] * xq[j];
    for (int c = lane; c < a; c += 32) {
        const int dof = act[c];
        s += E[(size_t)gw * a + c] * xpad[4 * (size_t)(dof / 3) + dof % 3];
    }
    s = wsum(s);
    if (lane == 0) yq[gw] = s;
}

// deterministic dots for the full residual: out = {|b - y|^2, |b|^2, b.x}
__global__ void residual_partial_kernel(const double* bf, const double* yf, const double* xf, int n4,
                                        const double* bq, const double* yq, const double* xq, int qm,
                                        double* part) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += gridDim.x * blockDim.x) {
        const double d = bf[e] - yf[e];
        s0 += d * d; s1 += bf[e] * bf[e]; s2 += bf[e] * xf[e];
    }
    if (blockIdx.x == 0)
        for (int e = threadIdx.x; e < qm; e += blockDim.x) {
            const double d = bq[e] - yq[e];
            s0 += d * d; s1 += bq[e] * bq[e]; s2 += bq[e] * xq[e];
        }
    s0 = bsum(s0);
    s1 = bsum(s1);
    s2 = bsum(s2);
    if (threadIdx.x == 0) {
        part[3 * blockIdx.x] = s0;
        part[3 * blockIdx.x + 1] = s1;
        part[3 * blockIdx.x + 2] = s2;
    }
}

// one warp: lane l sums partials l, l + 32, ... in order, then a fixed butterfly (deterministic)
__global__ void residual_final_kernel(const double* part, int np, double* out) {
    const int lane = threadIdx.x;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int i = lane; i < np; i += 32) { s0 += part[3 * i]; s1 += part[3 * i + 1]; s2 += part[3 * i + 2]; }
    s0 = wsum(s0); s1 = wsum(s1); s2 = wsum(s2);
    if (lane == 0) { out[0] = s0; out[1] = s1; out[2] = s2; }
}

// y (contiguous N) from node-padded y_f and yq
__global__ void scatter_y_kernel(const double* ypad, int n, int fo, const int* perm, const double* yq, int qm, int qo,
                                 double* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double* d = y + fo + 3 * (size_t)(perm ? perm[i] : i);
        d[0] = ypad[4 * (size_t)i];
        d[1] = ypad[4 * (size_t)i + 1];
        d[2] = ypad[4 * (size_t)i + 2];
    }
    if (i < qm) y[qo + i] = yq[i];
}

// x_acc += alpha * d (device alpha = min(1, num/den)); both contiguous N
__global__ void line_step_kernel(double* x, const double* d, int N, const double* nd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double num = nd[0], den = nd[1];
    const double alpha = (num > 0 && den > 0) ? fmin(1.0, num / den) : 0.0;
    x[i] += alpha * d[i];
}

__global__ void dot2_kernel(const double* a, const double* b, const double* c, int N, double* out) {
    // out[0] = a.b, out[1] = b.c  (one CTA, deterministic)
    double s0 = 0, s1 = 0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) { s0 += a[i] * b[i]; s1 += b[i] * c[i]; }
    s0 = bsum(s0);
    s1 = bsum(s1);
    if (threadIdx.x == 0) { out[0] = s0; out[1] = s1; }
}

__global__ void sub_kernel(const double* b, const double* y, double* r, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) r[i] = b[i] - y[i];
}

// FP64 copies of the coupled nodes' diagonal blocks; in the mixed modes the
// bulk planes drop them (they are applied in FP64 by the PCG kernel)
__global__ void split_active_diag_kernel(const int* act, int nact_nodes, const int* diag_pos, const double* v64,
                                         int nnz, float* vf, __nv_bfloat16* vb, double* dact) {
    const int an = blockIdx.x * blockDim.x + threadIdx.x;
    if (an >= nact_nodes) return;
    const int node = act[3 * an] / 3;
    const int k = diag_pos[node];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        const size_t o = (size_t)e * nnz + k;
        dact[9 * (size_t)an + e] = v64[o];
        if (vf) vf[o] = 0.0f;
        if (vb) vb[o] = __float2bfloat16_rn(0.0f);
    }
}

// dst[j * a + i] = src[j * a + perm[i]]: rows of an a x k column-major matrix reordered
__global__ void gather_rows_kernel(const double* src, int a, int k, const int* perm, double* dst) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= (long long)a * k) return;
    const int j = (int)(e / a), i = (int)(e - (long long)j * a);
    dst[e] = src[(size_t)j * a + perm[i]];
}

__global__ void f64_to_f32_kernel(const double* src, float* dst, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (float)src[i];
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

inline int blocks(long long n, int t = 256) { return (int)((n + t - 1) / t); }

}  // namespace

// ===========================================================================
// launchers
// ===========================================================================
void launch_pattern_hash(const int* rows, const int* cols, long long nnzb, unsigned long long* out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    const int g = (int)std::min<long long>(1184, std::max<long long>(1, (nnzb + 255) / 256));
    HSC_COUNTED(pattern_hash_kernel<<<g, 256, 0, st>>>(rows, cols, nnzb, out));
}

void launch_fill_bsr(const int* src, const double* values, int nnz, double* v64, float* vf, __nv_bfloat16* vb,
                     cudaStream_t st) {
    if (nnz == 0) return;
    HSC_COUNTED(fill_bsr_kernel<<<blocks(nnz), 256, 0, st>>>(src, values, nnz, v64, vf, vb));
}

void launch_dinv(int precision, const int* diag_pos, const double* v64, int nnz, int n, void* dinv, int* bad,
                 cudaStream_t st) {
    if (n == 0) return;
    if (precision == 0) HSC_COUNTED(dinv_kernel<double><<<blocks(n), 256, 0, st>>>(diag_pos, v64, nnz, n, (double*)dinv, bad));
    else HSC_COUNTED(dinv_kernel<float><<<blocks(n), 256, 0, st>>>(diag_pos, v64, nnz, n, (float*)dinv, bad));
}

void launch_extract(const int* qq, int nqq, const int* qf, int nqf, const double* values, int qm, int a, double* A,
                    double* E, int* node_nz, cudaStream_t st) {
    if (qm) cudaMemsetAsync(A, 0, sizeof(double) * qm * qm, st);
    if (qm && a) cudaMemsetAsync(E, 0, sizeof(double) * qm * a, st);
    if (a) cudaMemsetAsync(node_nz, 0, sizeof(int) * (a / 3), st);
    if (nqq) HSC_COUNTED(extract_A_kernel<<<blocks(nqq), 256, 0, st>>>(qq, nqq, values, qm, A));
    if (nqf) HSC_COUNTED(extract_E_kernel<<<blocks(nqf), 256, 0, st>>>(qf, nqf, values, a, E, node_nz));
}

cudaError_t launch_aca(const AcaParams& p, int grid, cudaStream_t st) {
    // column strips: a multiple of 32 columns per CTA, as few CTAs as cover the columns
    AcaParams q = p;
    const int strips = (p.nc + 31) / 32;
    // co-resident CTAs at this kernel's shared memory (m + a strip of doubles)
    const size_t smem_max = sizeof(double) * ((size_t)p.m + 32 * (size_t)strips);
    if (smem_max > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(aca_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)std::min<size_t>(smem_max, 227 * 1024));
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 1, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per = (strips + grid - 1) / grid;
    size_t smem = sizeof(double) * ((size_t)p.m + 32 * (size_t)per);
    for (;;) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, aca_kernel, 256, smem);
        const int cap = per_sm * sms;
        if (cap > 0 && (strips + per - 1) / per <= std::min(cap, grid)) break;
        if (per >= strips) return cudaErrorInvalidConfiguration;
        ++per;
        smem = sizeof(double) * ((size_t)p.m + 32 * (size_t)per);
    }
    q.strip = 32 * per;
    const int g = std::max(1, (p.nc + q.strip - 1) / q.strip);
    count_launch();
    void* args[] = {(void*)&q};
    const cudaError_t e = cudaLaunchCooperativeKernel((void*)aca_kernel, dim3(g), dim3(256), args, smem, st);
    debug_sync("aca_kernel");
    return e;
}

int aca_blocks_per_sm() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, aca_kernel, 256, 0);
    return b;
}

void launch_gemm(const GemmArgs& g, int M, int N, cudaStream_t st) {
    if (M <= 0 || N <= 0) return;
    dim3 grid((N + 31) / 32, (M + 31) / 32);
    HSC_COUNTED(gemm_kernel<<<grid, 128, 0, st>>>(g));
}

void launch_cholesky(const double* A, int m, double* L, int* bad, cudaStream_t st) {
    const size_t bytes = sizeof(double) * (size_t)m * m;
    const int use = bytes <= 200 * 1024;
    if (use) cudaFuncSetAttribute(cholesky_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    HSC_COUNTED(cholesky_kernel<<<1, 1024, use ? bytes : 0, st>>>(A, m, L, use, bad));
}

bool launch_chol_inverse(const double* A, int m, double* P, int* bad, cudaStream_t st, const int* dk) {
    if (m <= kGbMax) {
        HSC_COUNTED(gj_inverse_blocks_kernel<<<1, 1024, 0, st>>>(A, m, nullptr, nullptr, dk, P, bad));
        return true;
    }
    if (m <= kGjMax) {
        if (dk) HSC_COUNTED(gj_inverse_blocks_kernel<<<1, 1024, 0, st>>>(A, m, nullptr, nullptr, dk, P, bad));
        HSC_COUNTED(gj_inverse_reg_kernel<<<1, 512, 0, st>>>(A, m, dk, P, bad));
        return true;
    }
    const size_t bytes = sizeof(double) * ((size_t)m * (m + 1) + 2 * (size_t)m);
    if (bytes > 200 * 1024) return false;
    cudaFuncSetAttribute(gj_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    HSC_COUNTED(gj_inverse_kernel<<<1, 1024, bytes, st>>>(A, m, P, bad));
    return true;
}

bool launch_inverse_blocks(const double* A, int m, int nblk, int max_blk, const int* ptr, const int* idx, double* P,
                           int* bad, cudaStream_t st) {
    if (max_blk > kGbMax || nblk < 1) return false;
    cudaMemsetAsync(P, 0, sizeof(double) * (size_t)m * m, st);
    HSC_COUNTED(gj_inverse_blocks_kernel<<<nblk, 1024, 0, st>>>(A, m, ptr, idx, nullptr, P, bad));
    return true;
}

void launch_chol_solve(const double* L, int m, const double* B, int ldb, double* X, int ldx, int ncol,
                       const int* dncol, double* work, cudaStream_t st) {
    if (ncol <= 0) return;
    HSC_COUNTED(chol_solve_kernel<<<blocks((long long)ncol * 32), 256, 0, st>>>(L, m, B, ldb, X, ldx, ncol, dncol, work));
}

void launch_ldlt(double* C, int kmax, const int* dk, double* L, double* d, int* bad, cudaStream_t st) {
    const size_t bytes = sizeof(double) * (size_t)kmax * (kmax + 1);
    const int use = bytes <= 200 * 1024;
    if (use) cudaFuncSetAttribute(ldlt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // the register kernel for ranks up to 96, the shared-memory one beyond (each returns for the other's ranks)
    HSC_COUNTED(ldlt_reg_kernel<<<1, 1024, 0, st>>>(C, kmax, dk, L, d, bad));
    if (kmax > kGbMax) HSC_COUNTED(ldlt_kernel<<<1, 1024, use ? bytes : 0, st>>>(C, kmax, dk, L, d, use, bad));
}

void launch_block12_inverse(const double* A, int qm, double* Binv, int* bad, cudaStream_t st) {
    cudaMemsetAsync(Binv, 0, sizeof(double) * qm * qm, st);
    HSC_COUNTED(block12_inverse_kernel<<<blocks(qm / 12, 64), 64, 0, st>>>(A, qm, Binv, bad));
}

void launch_axpby_mat(double* Y, const double* X, double a, double b, int n, int diag_m, double diag_add,
                      cudaStream_t st) {
    HSC_COUNTED(axpby_mat_kernel<<<blocks(n), 256, 0, st>>>(Y, X, a, b, n, diag_m, diag_add));
}

void launch_symmetrize(double* P, int m, cudaStream_t st) { HSC_COUNTED(symmetrize_kernel<<<blocks((long long)m * m), 256, 0, st>>>(P, m)); }

void launch_frob(const double* X, int n, double* out, cudaStream_t st) { HSC_COUNTED(frob_kernel<<<1, 1024, 0, st>>>(X, n, out)); }

void launch_split_rhs(const double* b, int qo, int qm, int fo, int n, const int* perm, double* bq, double* bf,
                      cudaStream_t st) {
    HSC_COUNTED(split_rhs_kernel<<<blocks(std::max(qm, n)), 256, 0, st>>>(b, qo, qm, fo, n, perm, bq, bf));
}

void launch_wt_vec(const double* W, int qm, int kmax, const int* dk, const double* bq, double* c, cudaStream_t st) {
    if (kmax) HSC_COUNTED(wt_vec_kernel<<<blocks((long long)kmax * 32), 256, 0, st>>>(W, qm, kmax, dk, bq, c));
}

void launch_rhs_lowrank(const double* V, int a, const int* dk, const double* c, const int* act, double* rhs,
                        cudaStream_t st) {
    if (a) HSC_COUNTED(rhs_lowrank_kernel<<<blocks(a, 32), 32 * kColGroups, 0, st>>>(V, a, dk, c, act, rhs));
}

void launch_vt_x(const double* V, int a, int kmax, const int* dk, const int* act, const double* x, double* t,
                 cudaStream_t st) {
    if (kmax) HSC_COUNTED(vt_x_kernel<<<kmax, 256, 0, st>>>(V, a, dk, act, x, t));
}

void launch_backsub(const double* P, const double* W, int qm, int kmax, const int* dk, const double* bq,
                    const double* t, double* xq_out, double* xq_copy, cudaStream_t st) {
    if (qm) HSC_COUNTED(backsub_kernel<<<blocks((long long)qm * 32), 256, 0, st>>>(P, W, qm, kmax, dk, bq, t, xq_out, xq_copy));
}

void launch_scatter_x(const double* xpad, int n, int fo, const int* perm, double* xout, cudaStream_t st) {
    HSC_COUNTED(scatter_x_kernel<<<blocks(n), 256, 0, st>>>(xpad, n, fo, perm, xout));
}

void launch_gather_x(const double* x, int n, int fo, const int* perm, double* xpad, cudaStream_t st) {
    HSC_COUNTED(gather_x_kernel<<<blocks(n), 256, 0, st>>>(x, n, fo, perm, xpad));
}

void launch_full_spmv(const FullSpmv& f, cudaStream_t st) {
    if (f.bcoo_values)
        HSC_COUNTED(bcoo_row_spmv_kernel<<<blocks((long long)f.n * 4), 256, 0, st>>>(f.rowptr, f.colidx, f.src,
                                                                                  f.bcoo_values, f.n, f.xpad, f.ypad));
    else
        HSC_COUNTED(bsr_spmv64_kernel<<<blocks((long long)f.n * 4), 256, 0, st>>>(f.rowptr, f.colidx, f.v64, f.nnz, f.n,
                                                                               f.xpad, f.ypad));
    if (f.qm && f.a) HSC_COUNTED(et_xq_kernel<<<blocks(f.a, 32), 32 * kColGroups, 0, st>>>(f.E, f.qm, f.a, f.act, f.xq, f.ypad));
    if (f.qm && f.rowpart) {
        const int nchunk = abd_row_chunks(f.a);
        HSC_COUNTED(abd_rows_part_kernel<<<dim3(nchunk, (f.qm + 7) / 8), 256, 0, st>>>(f.A, f.E, f.qm, f.a, f.act, f.xq,
                                                                                      f.xpad, nchunk, f.rowpart));
        HSC_COUNTED(abd_rows_sum_kernel<<<blocks(f.qm), 256, 0, st>>>(f.rowpart, f.qm, nchunk, f.yq));
    } else if (f.qm)
        HSC_COUNTED(abd_rows_kernel<<<blocks((long long)f.qm * 32), 256, 0, st>>>(f.A, f.E, f.qm, f.a, f.act, f.xq, f.xpad,
                                                                      f.yq));
}

void launch_residual(const double* bf, const double* yf, const double* xf, int n, const double* bq, const double* yq,
                     const double* xq, int qm, double* part, int np, double* out, cudaStream_t st) {
    HSC_COUNTED(residual_partial_kernel<<<np, 256, 0, st>>>(bf, yf, xf, 4 * n, bq, yq, xq, qm, part));
    HSC_COUNTED(residual_final_kernel<<<1, 32, 0, st>>>(part, np, out));
}

void launch_scatter_y(const double* ypad, int n, int fo, const int* perm, const double* yq, int qm, int qo, double* y,
                      cudaStream_t st) {
    HSC_COUNTED(scatter_y_kernel<<<blocks(std::max(n, qm)), 256, 0, st>>>(ypad, n, fo, perm, yq, qm, qo, y));
}

void launch_line_step(double* x, const double* d, int N, const double* nd, cudaStream_t st) {
    HSC_COUNTED(line_step_kernel<<<blocks(N), 256, 0, st>>>(x, d, N, nd));
}

void launch_dot2(const double* a, const double* b, const double* c, int N, double* out, cudaStream_t st) {
    HSC_COUNTED(dot2_kernel<<<1, 1024, 0, st>>>(a, b, c, N, out));
}

void launch_sub(const double* b, const double* y, double* r, int N, cudaStream_t st) {
    HSC_COUNTED(sub_kernel<<<blocks(N), 256, 0, st>>>(b, y, r, N));
}

void launch_gather_rows(const double* src, int a, int k, const int* perm, double* dst, cudaStream_t st) {
    const long long n = (long long)a * k;
    if (n > 0) HSC_COUNTED(gather_rows_kernel<<<blocks(n), 256, 0, st>>>(src, a, k, perm, dst));
}

void launch_split_active_diag(const int* act, int nact_nodes, const int* diag_pos, const double* v64, int nnz,
                              float* vf, __nv_bfloat16* vb, double* dact, cudaStream_t st) {
    if (nact_nodes <= 0) return;
    HSC_COUNTED(split_active_diag_kernel<<<blocks(nact_nodes), 256, 0, st>>>(act, nact_nodes, diag_pos, v64, nnz, vf,
                                                                              vb, dact));
}

void read_fail_setup(long long* out) { hsc_read_fail(out); }

void convert_f64_f32(const double* src, float* dst, long long n, cudaStream_t st) {
    if (n > 0) HSC_COUNTED(f64_to_f32_kernel<<<blocks(n), 256, 0, st>>>(src, dst, n));
}

void set_int(int* p, int v, cudaStream_t st) { HSC_COUNTED(set_int_kernel<<<1, 1, 0, st>>>(p, v)); }

}  // namespace hsc
