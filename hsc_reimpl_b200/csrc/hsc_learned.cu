// Learned polynomial preconditioner.
//
// The preconditioner of the Schur PCG is z = sum_k w_k t_k with
// t_0 = w Dd^-1 r and t_k = t_{k-1} - w Dd^-1 S t_{k-1} (the Schur basis), so
// for an eigenvalue mu of G = w Dd^-1 S the preconditioned operator has the
// eigenvalue lambda(mu) = mu q(mu), q(mu) = sum_k w_k (1 - mu)^k.  The
// reference fixes w_k = 1 (the Neumann series, linear_hsc.cu:330-343); here a
// small MLP chooses the 8 weights per system from 16 spectral features.
//
//   features  (in a solve, device only): statistics of the Jacobi-scaled FEM
//             operator (off-diagonal mass |D_ii^-1 D_ij|_F per block row,
//             spread of the diagonal stiffness), the share of the coupled
//             rows' stiffness that the low-rank term V C V^T removes, and the
//             previous solve's Lanczos extremes of the same system;
//   MLP       16 -> 64 -> 64 -> 8, ReLU, softplus outputs (positive weights);
//             BF16 parameters, FP32 accumulation in a fixed order;
//   training  (hsc_mlp_forward / hsc_mlp_backward / hsc_poly_ls_loss /
//             hsc_adam_step): the loss of one system is the least-squares
//             residual polynomial on the spectral measure of G seen from the
//             system's right-hand side (Ritz values theta_i and weights tau_i
//             of a short Lanczos run of the solver):
//                 L(w) = sum_i tau_i (1 - theta_i q_w(theta_i))^2.
//             Batch reductions of the parameter gradients run one thread per
//             parameter over the samples in order: bit-reproducible.
#include <cuda_bf16.h>

#include "../../include/hsc_c_api.h"
#include "hsc_learned.cuh"

namespace hsc {

namespace {

__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

__device__ __forceinline__ uint16_t f2bf(float f) {
    const __nv_bfloat16 h = __float2bfloat16_rn(f);
    return *reinterpret_cast<const uint16_t*>(&h);
}

__device__ __forceinline__ float softplus(float o) { return o > 20.f ? o : log1pf(expf(o)); }
__device__ __forceinline__ float sigmoid(float o) { return 1.f / (1.f + expf(-o)); }

// ---------------------------------------------------------------------------
// features
// ---------------------------------------------------------------------------
// partial layout: 0 sum off, 1 sum off^2, 2 max off, 3 count(off > 1),
// 4 min log10 tr, 5 max log10 tr, 6 sum log10 tr, 7 sum (log10 tr)^2,
// 8 sum off at coupled nodes, 9 coupled nodes, 10 sum tr at coupled nodes,
// 11 rows counted
enum { P_SUM = 0, P_SQ, P_MAX, P_CNT, P_LMIN, P_LMAX, P_LSUM, P_LSQ, P_ASUM, P_ACNT, P_ATR, P_ROWS, P_N };
static_assert(P_N <= kFeatParts, "partial layout");

__device__ __forceinline__ double red_op(int j, double a, double b) {
    if (j == P_MAX || j == P_LMAX) return fmax(a, b);
    if (j == P_LMIN) return fmin(a, b);
    return a + b;
}

__device__ __forceinline__ double red_init(int j) {
    if (j == P_MAX || j == P_LMAX) return -1e300;
    if (j == P_LMIN) return 1e300;
    return 0.0;
}

__global__ void feat_rows_kernel(const FeatArgs f) {
    double acc[P_N];
#pragma unroll
    for (int j = 0; j < P_N; ++j) acc[j] = red_init(j);
    const size_t nz = (size_t)f.nnz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < f.n; i += gridDim.x * blockDim.x) {
        const int kd = f.diag_pos[i];
        double d[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) d[e] = f.v64[e * nz + kd];
        const double c00 = d[4] * d[8] - d[5] * d[7], c01 = d[5] * d[6] - d[3] * d[8], c02 = d[3] * d[7] - d[4] * d[6];
        const double det = d[0] * c00 + d[1] * c01 + d[2] * c02;
        const double tr = d[0] + d[4] + d[8];
        double off = 0.0;
        if (det > 0 && isfinite(det)) {
            const double id = 1.0 / det;
            double inv[9];
            inv[0] = c00 * id; inv[1] = (d[2] * d[7] - d[1] * d[8]) * id; inv[2] = (d[1] * d[5] - d[2] * d[4]) * id;
            inv[3] = c01 * id; inv[4] = (d[0] * d[8] - d[2] * d[6]) * id; inv[5] = (d[2] * d[3] - d[0] * d[5]) * id;
            inv[6] = c02 * id; inv[7] = (d[1] * d[6] - d[0] * d[7]) * id; inv[8] = (d[0] * d[4] - d[1] * d[3]) * id;
            for (int k = f.rowptr[i]; k < f.rowptr[i + 1]; ++k) {
                if (k == kd) continue;
                double b[9];
#pragma unroll
                for (int e = 0; e < 9; ++e) b[e] = f.v64[e * nz + k];
                double s = 0.0;
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double m = inv[3 * r] * b[c] + inv[3 * r + 1] * b[3 + c] + inv[3 * r + 2] * b[6 + c];
                        s += m * m;
                    }
                off += sqrt(s);
            }
        }
        const double lt = tr > 0 ? log10(tr) : 0.0;
        acc[P_SUM] += off;
        acc[P_SQ] += off * off;
        acc[P_MAX] = fmax(acc[P_MAX], off);
        acc[P_CNT] += off > 1.0 ? 1.0 : 0.0;
        acc[P_LMIN] = fmin(acc[P_LMIN], lt);
        acc[P_LMAX] = fmax(acc[P_LMAX], lt);
        acc[P_LSUM] += lt;
        acc[P_LSQ] += lt * lt;
        if (f.rowflag[i] >= 0) {
            acc[P_ASUM] += off;
            acc[P_ACNT] += 1.0;
            acc[P_ATR] += tr;
        }
        acc[P_ROWS] += 1.0;
    }
    // fixed-order block reduction: warp shuffles, then warp results in order
    __shared__ double s_part[32][P_N];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < P_N; ++j) {
        double v = acc[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = red_op(j, v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) s_part[warp][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < P_N) {
        const int j = threadIdx.x;
        double v = red_init(j);
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = red_op(j, v, s_part[w][j]);
        f.part[(size_t)blockIdx.x * kFeatParts + j] = v;
    }
}

__device__ __forceinline__ float clampf(double v) {
    if (!isfinite(v)) return 0.f;
    return (float)fmin(8.0, fmax(-8.0, v));
}

// one block: reduce the partials, the low-rank trace, assemble the features,
// then (optionally) the MLP for this one system
__global__ void __launch_bounds__(256) feat_final_kernel(const FeatArgs f) {
    __shared__ double s_red[P_N];
    __shared__ double s_lr[kMaxRank];
    __shared__ float s_f[kFeat];
    __shared__ float s_h1[kHidden], s_h2[kHidden];
    const int t = threadIdx.x;
    if (t < P_N) {
        double v = red_init(t);
        for (int b = 0; b < f.nparts; ++b) v = red_op(t, v, f.part[(size_t)b * kFeatParts + t]);
        s_red[t] = v;
    }
    const int rank = min(*f.rank, min(f.kmax, kMaxRank));
    for (int j = t; j < kMaxRank; j += blockDim.x) {
        double s = 0.0;
        if (j < rank) {
            const double* col = f.vt64 + (size_t)j * f.a;
            for (int i = 0; i < f.a; ++i) s += col[i] * col[i];
            s *= f.dpiv[j];
        }
        s_lr[j] = s;
    }
    __syncthreads();
    if (t == 0) {
        double lr = 0.0;
        for (int j = 0; j < rank; ++j) lr += s_lr[j];
        const double rows = fmax(1.0, s_red[P_ROWS]);
        const double mean = s_red[P_SUM] / rows;
        const double var = fmax(0.0, s_red[P_SQ] / rows - mean * mean);
        const double lmean = s_red[P_LSUM] / rows;
        const double lvar = fmax(0.0, s_red[P_LSQ] / rows - lmean * lmean);
        const double acnt = s_red[P_ACNT];
        const double rho = s_red[P_ATR] > 0 ? lr / s_red[P_ATR] : 0.0;
        const double* pv = f.prev;
        const bool has = pv[0] > 0.5;
        s_f[0] = clampf(log10(fmax(1.0, (double)f.n)) / 5.0);
        s_f[1] = clampf(10.0 * f.a / fmax(1.0, 3.0 * f.n));
        s_f[2] = clampf(rank / 128.0);
        s_f[3] = clampf(mean);
        s_f[4] = clampf(sqrt(var));
        s_f[5] = clampf(s_red[P_MAX] / 4.0);
        s_f[6] = clampf(s_red[P_CNT] / rows);
        s_f[7] = clampf((s_red[P_LMAX] - s_red[P_LMIN]) / 10.0);
        s_f[8] = clampf(sqrt(lvar) / 3.0);
        s_f[9] = clampf(acnt > 0 ? s_red[P_ASUM] / acnt : 0.0);
        s_f[10] = clampf(rho);
        s_f[11] = clampf(log10(fmax(1.0 - rho, 1e-12)) / 6.0);
        s_f[12] = has ? 1.f : 0.f;
        s_f[13] = has ? clampf(log10(fmax(pv[1] / fmax(pv[4], 1e-30), 1e-30)) / 6.0) : 0.f;
        s_f[14] = has ? clampf(log10(fmax(pv[2], 1e-30))) : 0.f;
        s_f[15] = has ? clampf(log10(fmax(pv[3], 1.0)) / 4.0) : 0.f;
    }
    __syncthreads();
    if (t < kFeat) f.feat[t] = s_f[t];
    if (!f.mlp) return;
    const uint16_t* P = f.mlp;
    if (t < kHidden) {
        float s = bf2f(P[kOffB1 + t]);
        for (int i = 0; i < kFeat; ++i) s += bf2f(P[kOffW1 + t * kFeat + i]) * s_f[i];
        s_h1[t] = fmaxf(s, 0.f);
    }
    __syncthreads();
    if (t < kHidden) {
        float s = bf2f(P[kOffB2 + t]);
        for (int i = 0; i < kHidden; ++i) s += bf2f(P[kOffW2 + t * kHidden + i]) * s_h1[i];
        s_h2[t] = fmaxf(s, 0.f);
    }
    __syncthreads();
    if (t < kPolyOut) {
        float s = bf2f(P[kOffB3 + t]);
        for (int i = 0; i < kHidden; ++i) s += bf2f(P[kOffW3 + t * kHidden + i]) * s_h2[i];
        f.w[t] = (double)softplus(s);
    }
}

// ---------------------------------------------------------------------------
// training kernels
// ---------------------------------------------------------------------------
constexpr int kTrainThreads = 256;
constexpr int kTrainWarps = kTrainThreads / 32;

// forward, one warp per sample; lane o computes outputs o and o + 32
__global__ void __launch_bounds__(kTrainThreads) mlp_fwd_kernel(const uint16_t* __restrict__ P,
                                                               const float* __restrict__ X, int B, float* H1,
                                                               float* H2, float* O, float* W) {
    __shared__ float w1t[kFeat][kHidden], w2t[kHidden][kHidden], w3t[kHidden][kPolyOut];
    __shared__ float b1[kHidden], b2[kHidden], b3[kPolyOut];
    __shared__ float xs[kTrainWarps][kFeat], h1s[kTrainWarps][kHidden], h2s[kTrainWarps][kHidden];
    for (int e = threadIdx.x; e < kHidden * kFeat; e += kTrainThreads) w1t[e % kFeat][e / kFeat] = bf2f(P[kOffW1 + e]);
    for (int e = threadIdx.x; e < kHidden * kHidden; e += kTrainThreads)
        w2t[e % kHidden][e / kHidden] = bf2f(P[kOffW2 + e]);
    for (int e = threadIdx.x; e < kPolyOut * kHidden; e += kTrainThreads)
        w3t[e % kHidden][e / kHidden] = bf2f(P[kOffW3 + e]);
    for (int e = threadIdx.x; e < kHidden; e += kTrainThreads) { b1[e] = bf2f(P[kOffB1 + e]); b2[e] = bf2f(P[kOffB2 + e]); }
    if (threadIdx.x < kPolyOut) b3[threadIdx.x] = bf2f(P[kOffB3 + threadIdx.x]);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s = blockIdx.x * kTrainWarps + warp; s < B; s += gridDim.x * kTrainWarps) {
        if (lane < kFeat) xs[warp][lane] = X[(size_t)s * kFeat + lane];
        __syncwarp();
        for (int o = lane; o < kHidden; o += 32) {
            float a = b1[o];
            for (int i = 0; i < kFeat; ++i) a += w1t[i][o] * xs[warp][i];
            a = fmaxf(a, 0.f);
            h1s[warp][o] = a;
            if (H1) H1[(size_t)s * kHidden + o] = a;
        }
        __syncwarp();
        for (int o = lane; o < kHidden; o += 32) {
            float a = b2[o];
            for (int i = 0; i < kHidden; ++i) a += w2t[i][o] * h1s[warp][i];
            a = fmaxf(a, 0.f);
            h2s[warp][o] = a;
            if (H2) H2[(size_t)s * kHidden + o] = a;
        }
        __syncwarp();
        if (lane < kPolyOut) {
            float a = b3[lane];
            for (int i = 0; i < kHidden; ++i) a += w3t[i][lane] * h2s[warp][i];
            if (O) O[(size_t)s * kPolyOut + lane] = a;
            if (W) W[(size_t)s * kPolyOut + lane] = softplus(a);
        }
        __syncwarp();
    }
}

// backward through the layers, one warp per sample: gradients of the
// pre-activations (GO = dL/do, GZ2, GZ1) from GW = dL/dw
__global__ void __launch_bounds__(kTrainThreads) mlp_bwd_sample_kernel(const uint16_t* __restrict__ P,
                                                                      const float* __restrict__ H1,
                                                                      const float* __restrict__ H2,
                                                                      const float* __restrict__ O,
                                                                      const float* __restrict__ GW, int B, float* GO,
                                                                      float* GZ2, float* GZ1) {
    __shared__ float w2[kHidden][kHidden], w3[kPolyOut][kHidden];
    __shared__ float gos[kTrainWarps][kPolyOut], gz2s[kTrainWarps][kHidden];
    for (int e = threadIdx.x; e < kHidden * kHidden; e += kTrainThreads) w2[e / kHidden][e % kHidden] = bf2f(P[kOffW2 + e]);
    for (int e = threadIdx.x; e < kPolyOut * kHidden; e += kTrainThreads) w3[e / kHidden][e % kHidden] = bf2f(P[kOffW3 + e]);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s = blockIdx.x * kTrainWarps + warp; s < B; s += gridDim.x * kTrainWarps) {
        if (lane < kPolyOut) {
            const float g = GW[(size_t)s * kPolyOut + lane] * sigmoid(O[(size_t)s * kPolyOut + lane]);
            gos[warp][lane] = g;
            GO[(size_t)s * kPolyOut + lane] = g;
        }
        __syncwarp();
        for (int j = lane; j < kHidden; j += 32) {
            float g = 0.f;
            for (int o = 0; o < kPolyOut; ++o) g += w3[o][j] * gos[warp][o];
            g = H2[(size_t)s * kHidden + j] > 0.f ? g : 0.f;
            gz2s[warp][j] = g;
            GZ2[(size_t)s * kHidden + j] = g;
        }
        __syncwarp();
        for (int i = lane; i < kHidden; i += 32) {
            float g = 0.f;
            for (int j = 0; j < kHidden; ++j) g += w2[j][i] * gz2s[warp][j];
            GZ1[(size_t)s * kHidden + i] = H1[(size_t)s * kHidden + i] > 0.f ? g : 0.f;
        }
        __syncwarp();
    }
}

// parameter gradients: one thread per parameter, samples summed in order
__global__ void mlp_bwd_weight_kernel(const float* __restrict__ X, const float* __restrict__ H1,
                                      const float* __restrict__ H2, const float* __restrict__ GO,
                                      const float* __restrict__ GZ2, const float* __restrict__ GZ1, int B,
                                      float* __restrict__ G) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float* gsrc;
    const float* asrc = nullptr;
    int gs, go_, as = 0, ao = 0;
    if (p < kOffB1) { const int o = p / kFeat, i = p % kFeat; gsrc = GZ1; gs = kHidden; go_ = o; asrc = X; as = kFeat; ao = i; }
    else if (p < kOffW2) { gsrc = GZ1; gs = kHidden; go_ = p - kOffB1; }
    else if (p < kOffB2) { const int q = p - kOffW2, o = q / kHidden, i = q % kHidden; gsrc = GZ2; gs = kHidden; go_ = o; asrc = H1; as = kHidden; ao = i; }
    else if (p < kOffW3) { gsrc = GZ2; gs = kHidden; go_ = p - kOffB2; }
    else if (p < kOffB3) { const int q = p - kOffW3, o = q / kHidden, i = q % kHidden; gsrc = GO; gs = kPolyOut; go_ = o; asrc = H2; as = kHidden; ao = i; }
    else { gsrc = GO; gs = kPolyOut; go_ = p - kOffB3; }
    float acc = 0.f;
    if (asrc)
        for (int s = 0; s < B; ++s) acc += gsrc[(size_t)s * gs + go_] * asrc[(size_t)s * as + ao];
    else
        for (int s = 0; s < B; ++s) acc += gsrc[(size_t)s * gs + go_];
    G[p] = acc;
}

// L = scale * sum_i tau_i (1 - theta_i q_w(theta_i))^2 per sample, and dL/dw
__global__ void poly_ls_loss_kernel(const float* __restrict__ W, const float* __restrict__ TH,
                                    const float* __restrict__ TAU, int B, int m, float scale, float* loss,
                                    float* GW) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    float w[kPolyOut], g[kPolyOut];
#pragma unroll
    for (int k = 0; k < kPolyOut; ++k) { w[k] = W[(size_t)s * kPolyOut + k]; g[k] = 0.f; }
    float L = 0.f;
    for (int i = 0; i < m; ++i) {
        const float th = TH[(size_t)s * m + i], ta = TAU[(size_t)s * m + i];
        float basis[kPolyOut];
        float pw = th, lam = 0.f;
#pragma unroll
        for (int k = 0; k < kPolyOut; ++k) {
            basis[k] = pw;
            lam += w[k] * pw;
            pw *= 1.f - th;
        }
        const float r = 1.f - lam;
        L += ta * r * r;
#pragma unroll
        for (int k = 0; k < kPolyOut; ++k) g[k] -= 2.f * ta * r * basis[k];
    }
    if (loss) loss[s] = L * scale;
#pragma unroll
    for (int k = 0; k < kPolyOut; ++k) GW[(size_t)s * kPolyOut + k] = g[k] * scale;
}

__global__ void adam_kernel(float* master, uint16_t* P, const float* G, float* M, float* V, int n, float lr,
                            float b1, float b2, float eps, float wd, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i] + wd * master[i];
    const float m = b1 * M[i] + (1.f - b1) * g;
    const float v = b2 * V[i] + (1.f - b2) * g * g;
    M[i] = m;
    V[i] = v;
    const float w = master[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    master[i] = w;
    P[i] = f2bf(w);
}

int status_of(cudaError_t e) { return e == cudaSuccess ? HSC_OK : HSC_ERR_CUDA; }

}  // namespace

cudaError_t launch_features(const FeatArgs& f, cudaStream_t st) {
    if (f.n <= 0 || f.nparts <= 0) return cudaSuccess;
    count_launch();
    feat_rows_kernel<<<f.nparts, 256, 0, st>>>(f);
    count_launch();
    feat_final_kernel<<<1, 256, 0, st>>>(f);
    debug_sync("features");
    return cudaGetLastError();
}

}  // namespace hsc

using namespace hsc;

extern "C" {

int hsc_mlp_forward(const uint16_t* d_params, const float* d_x, int32_t batch, float* d_h1, float* d_h2,
                    float* d_o, float* d_w, void* stream) {
    if (!d_params || !d_x || batch < 0) return HSC_ERR_INVALID;
    if (batch == 0) return HSC_OK;
    const int grid = (batch + kTrainWarps - 1) / kTrainWarps;
    count_launch();
    mlp_fwd_kernel<<<grid < 1184 ? grid : 1184, kTrainThreads, 0, (cudaStream_t)stream>>>(d_params, d_x, batch, d_h1,
                                                                                         d_h2, d_o, d_w);
    return status_of(cudaGetLastError());
}

int hsc_mlp_backward(const uint16_t* d_params, const float* d_x, const float* d_h1, const float* d_h2,
                     const float* d_o, const float* d_gw, int32_t batch, float* d_scratch, float* d_grad,
                     void* stream) {
    if (!d_params || !d_x || !d_h1 || !d_h2 || !d_o || !d_gw || !d_scratch || !d_grad || batch < 1)
        return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    float* go = d_scratch;
    float* gz2 = go + (size_t)batch * kPolyOut;
    float* gz1 = gz2 + (size_t)batch * kHidden;
    const int grid = (batch + kTrainWarps - 1) / kTrainWarps;
    count_launch();
    mlp_bwd_sample_kernel<<<grid < 1184 ? grid : 1184, kTrainThreads, 0, st>>>(d_params, d_h1, d_h2, d_o, d_gw,
                                                                                batch, go, gz2, gz1);
    count_launch();
    mlp_bwd_weight_kernel<<<(kParams + 127) / 128, 128, 0, st>>>(d_x, d_h1, d_h2, go, gz2, gz1, batch, d_grad);
    return status_of(cudaGetLastError());
}

int hsc_poly_ls_loss(const float* d_w, const float* d_theta, const float* d_tau, int32_t batch, int32_t m,
                     float scale, float* d_loss, float* d_gw, void* stream) {
    if (!d_w || !d_theta || !d_tau || !d_gw || batch < 0 || m < 1) return HSC_ERR_INVALID;
    if (batch == 0) return HSC_OK;
    count_launch();
    poly_ls_loss_kernel<<<(batch + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_w, d_theta, d_tau, batch, m, scale,
                                                                             d_loss, d_gw);
    return status_of(cudaGetLastError());
}

int hsc_adam_step(float* d_master, uint16_t* d_params, const float* d_grad, float* d_m, float* d_v, int32_t n,
                  float lr, float beta1, float beta2, float eps, float weight_decay, int32_t step, void* stream) {
    if (!d_master || !d_params || !d_grad || !d_m || !d_v || n < 1 || step < 1) return HSC_ERR_INVALID;
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    count_launch();
    adam_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_master, d_params, d_grad, d_m, d_v, n, lr, beta1,
                                                                 beta2, eps, weight_decay, c1, c2);
    return status_of(cudaGetLastError());
}

}  // extern "C"
