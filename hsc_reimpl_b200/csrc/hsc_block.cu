// Block-local Woodbury preconditioner and pipelined Schur PCG (see hsc_block.cuh).
#include <algorithm>
#include <type_traits>

#include "../../include/hsc_c_api.h"
#include "hsc_block.cuh"
#include "hsc_check.cuh"
#include "hsc_setup.cuh"

namespace hsc {

namespace {

template <class MT> struct BlkDinv { using T = float; };
template <> struct BlkDinv<double> { using T = double; };

__device__ __forceinline__ double bwarp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// o = s * (B r) with B the 3x3 block of row `lr` among 9 planes of stride `stride`
template <class DT>
__device__ __forceinline__ void blk_dinv(const DT* sd, int stride, int lr, double s, double r0, double r1, double r2,
                                         double& o0, double& o1, double& o2) {
    const DT* d = sd + lr;
    o0 = s * ((double)d[0] * r0 + (double)d[stride] * r1 + (double)d[2 * stride] * r2);
    o1 = s * ((double)d[3 * stride] * r0 + (double)d[4 * stride] * r1 + (double)d[5 * stride] * r2);
    o2 = s * ((double)d[6 * stride] * r0 + (double)d[7 * stride] * r1 + (double)d[8 * stride] * r2);
}

// ---------------------------------------------------------------------------
// columns of each coupling component: the body of U[:, j]'s first nonzero row
// gives its component; counting sort into comp_col_ptr / comp_cols (one CTA)
// ---------------------------------------------------------------------------
__global__ void block_columns_kernel(BlockPlan p) {
    __shared__ int s_cnt[257];
    const int k = *p.rank;
    for (int g = threadIdx.x; g <= p.ncomp; g += blockDim.x) s_cnt[g] = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < p.kmax; j += blockDim.x) {
        int comp = -1;
        if (j < k)
            for (int i = 0; i < p.qm; ++i)
                if (p.U[(size_t)j * p.qm + i] != 0.0) { comp = p.comp_of_body[i / 12]; break; }
        p.comp_of_col[j] = comp;
        if (comp >= 0) atomicAdd(&s_cnt[comp + 1], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int g = 0; g < p.ncomp; ++g) s_cnt[g + 1] += s_cnt[g];
        for (int g = 0; g <= p.ncomp; ++g) p.comp_col_ptr[g] = s_cnt[g];
        // columns in increasing order inside each component (deterministic)
        for (int j = 0; j < k; ++j) {
            const int comp = p.comp_of_col[j];
            if (comp >= 0) p.comp_cols[s_cnt[comp]++] = j;
        }
    }
}

// ---------------------------------------------------------------------------
// the CTA's column list: the columns of the components in its part, with the
// CTA's contributor slot for each
// ---------------------------------------------------------------------------
__device__ int build_cols(const BlockPlan& p, int cta, int* s_cols, int* s_slot) {
    __shared__ int s_n;
    if (threadIdx.x == 0) {
        int nc = 0;
        for (int e = p.cta_comp_ptr[cta]; e < p.cta_comp_ptr[cta + 1]; ++e) {
            const int g = p.cta_comp[e], slot = p.cta_comp_slot[e];
            for (int q = p.comp_col_ptr[g]; q < p.comp_col_ptr[g + 1] && nc < p.kmax; ++q) {
                s_cols[nc] = p.comp_cols[q];
                s_slot[nc] = slot;
                ++nc;
            }
        }
        s_n = nc;
    }
    __syncthreads();
    return s_n;
}

// ---------------------------------------------------------------------------
// shared-memory staging of a CTA's rows: local row pointers, window positions of
// the blocks' columns, value planes (when staged), Dd^-1 planes, window node ids
// ---------------------------------------------------------------------------
template <class MT>
struct Slice {
    int rb, re, R, kb0, nblk, wn0, nwin, wown, ab, ae, na;
    int* rp;
    unsigned short* lc;
    const MT* val;        // planes, stride pstride (shared or global)
    size_t pstride;
    const typename BlkDinv<MT>::T* dinv;  // planes, stride R
    int* wn;
};

template <class MT>
__device__ Slice<MT> stage_slice(const BlockPlan& p, int cta, unsigned char* sm) {
    using DT = typename BlkDinv<MT>::T;
    Slice<MT> s;
    s.rb = p.cta_row[2 * cta];
    s.re = p.cta_row[2 * cta + 1];
    s.R = s.re - s.rb;
    s.kb0 = __ldg(p.rowptr + s.rb);
    s.nblk = __ldg(p.rowptr + s.re) - s.kb0;
    s.wn0 = p.win_off[cta];
    s.nwin = p.win_off[cta + 1] - s.wn0;
    s.wown = p.win_own[cta];
    s.ab = p.cta_act[2 * cta];
    s.ae = p.cta_act[2 * cta + 1];
    s.na = s.ae - s.ab;
    s.rp = reinterpret_cast<int*>(sm + p.off_rp);
    s.lc = reinterpret_cast<unsigned short*>(sm + p.off_lc);
    s.wn = reinterpret_cast<int*>(sm + p.off_wn);
    DT* sd = reinterpret_cast<DT*>(sm + p.off_dinv);
    const MT* vals = reinterpret_cast<const MT*>(p.vals);
    const DT* dinv = reinterpret_cast<const DT*>(p.dinv);
    for (int e = threadIdx.x; e <= s.R; e += blockDim.x) s.rp[e] = __ldg(p.rowptr + s.rb + e) - s.kb0;
    for (int e = threadIdx.x; e < s.nblk; e += blockDim.x) s.lc[e] = p.lcol[s.kb0 + e];
    for (int e = threadIdx.x; e < s.nwin; e += blockDim.x) s.wn[e] = p.win_nodes[s.wn0 + e];
    for (int e = threadIdx.x; e < 9 * s.R; e += blockDim.x) {
        const int pl = e / s.R, lr = e - pl * s.R;
        sd[e] = dinv[(size_t)pl * p.n + s.rb + lr];
    }
    if (p.stage_vals) {
        MT* sv = reinterpret_cast<MT*>(sm + p.off_val);
        for (int e = threadIdx.x; e < 9 * s.nblk; e += blockDim.x) {
            const int pl = e / s.nblk, kl = e - pl * s.nblk;
            sv[e] = vals[(size_t)pl * p.nnz + s.kb0 + kl];
        }
        s.val = sv;
        s.pstride = (size_t)s.nblk;
    } else {
        s.val = vals + s.kb0;
        s.pstride = (size_t)p.nnz;
    }
    s.dinv = sd;
    __syncthreads();
    return s;
}

template <class MT>
__device__ __forceinline__ double ldv(const Slice<MT>& s, size_t off, bool global) {
    return global ? (double)__ldg(s.val + off) : (double)s.val[off];
}

// y_row = sum over the row's blocks B x[col], four threads per row, for the
// CTA's own rows.  `local` restricts to the blocks whose column is an own row
// (D_loc) and then reads x from the own-row vector xo (3 per row); otherwise x
// comes from the staged window xw (4 per window node).  Fixed summation order.
template <class MT, class Epi>
__device__ __forceinline__ void slice_spmv(const Slice<MT>& s, bool gvals, bool local, const double* xo,
                                           const double* xw, Epi& epi) {
    const int sub = threadIdx.x & 3;
    for (int lr0 = 0; lr0 < s.R; lr0 += blockDim.x / 4) {
        const int lr = lr0 + (threadIdx.x >> 2);
        double a0 = 0, a1 = 0, a2 = 0;
        if (lr < s.R) {
            const int k1 = s.rp[lr + 1];
            for (int kk = s.rp[lr] + sub; kk < k1; kk += 4) {
                const int w = s.lc[kk];
                double x0, x1, x2;
                if (local) {
                    const int ol = w - s.wown;
                    if (ol < 0 || ol >= s.R) continue;
                    x0 = xo[3 * ol]; x1 = xo[3 * ol + 1]; x2 = xo[3 * ol + 2];
                } else {
                    x0 = xw[4 * w]; x1 = xw[4 * w + 1]; x2 = xw[4 * w + 2];
                }
                const size_t o = kk, ps = s.pstride;
                a0 += ldv(s, o, gvals) * x0 + ldv(s, o + ps, gvals) * x1 + ldv(s, o + 2 * ps, gvals) * x2;
                a1 += ldv(s, o + 3 * ps, gvals) * x0 + ldv(s, o + 4 * ps, gvals) * x1 + ldv(s, o + 5 * ps, gvals) * x2;
                a2 += ldv(s, o + 6 * ps, gvals) * x0 + ldv(s, o + 7 * ps, gvals) * x1 + ldv(s, o + 8 * ps, gvals) * x2;
            }
        }
        a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 1);
        a0 += __shfl_xor_sync(0xffffffffu, a0, 2);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 2);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 2);
        if (lr < s.R && sub == 0) epi(lr, a0, a1, a2);
    }
}

// the FP64 diagonal block of a coupled node (mixed modes keep it out of the planes)
__device__ __forceinline__ void add_dact(const BlockPlan& p, int node, double x0, double x1, double x2, double& y0,
                                         double& y1, double& y2) {
    const int an = p.rowflag[node];
    if (an < 0) return;
    const double* d = p.dact + 9 * (size_t)an;
    y0 += d[0] * x0 + d[1] * x1 + d[2] * x2;
    y1 += d[3] * x0 + d[4] * x1 + d[5] * x2;
    y2 += d[6] * x0 + d[7] * x1 + d[8] * x2;
}

__device__ __forceinline__ double poly_weight(const BlockPlan& p, int k) { return p.wdev ? p.wdev[k] : p.w[k]; }

// z = L v over the CTA's rows (v, z, t, u: 3 R doubles in shared memory; t and u
// are scratch).  Each term is one local SpMV; no grid barrier.
template <class MT>
__device__ void local_poly(const BlockPlan& p, const Slice<MT>& s, bool split, const double* v, double* z, double* t,
                           double* u) {
    using DT = typename BlkDinv<MT>::T;
    const bool gv = !p.stage_vals;
    const double w0 = poly_weight(p, 0);
    for (int e = threadIdx.x; e < s.R; e += blockDim.x) {
        double o0, o1, o2;
        blk_dinv<DT>(s.dinv, s.R, e, p.omega, v[3 * e], v[3 * e + 1], v[3 * e + 2], o0, o1, o2);
        t[3 * e] = o0; t[3 * e + 1] = o1; t[3 * e + 2] = o2;
        z[3 * e] = w0 * o0; z[3 * e + 1] = w0 * o1; z[3 * e + 2] = w0 * o2;
    }
    __syncthreads();
    double* tc = t;
    double* tn = u;
    for (int k = 1; k < p.nterms; ++k) {
        const double wk = poly_weight(p, k);
        auto epi = [&](int lr, double y0, double y1, double y2) {
            const double c0 = tc[3 * lr], c1 = tc[3 * lr + 1], c2 = tc[3 * lr + 2];
            if (split) add_dact(p, s.rb + lr, c0, c1, c2, y0, y1, y2);
            double e0, e1, e2;
            blk_dinv<DT>(s.dinv, s.R, lr, p.omega, y0, y1, y2, e0, e1, e2);
            const double n0 = c0 - e0, n1 = c1 - e1, n2 = c2 - e2;
            tn[3 * lr] = n0; tn[3 * lr + 1] = n1; tn[3 * lr + 2] = n2;
            z[3 * lr] += wk * n0; z[3 * lr + 1] += wk * n1; z[3 * lr + 2] += wk * n2;
        };
        slice_spmv<MT>(s, gv, true, tc, nullptr, epi);
        __syncthreads();
        double* tmp = tc; tc = tn; tn = tmp;
    }
}

// the same polynomial on NB vectors at once (column c of an NB-batch at offset
// c * 3 p.R): one pass over the blocks per term serves all NB
template <class MT, int NB>
__device__ void local_poly_multi(const BlockPlan& p, const Slice<MT>& s, bool split, const double* v, double* z,
                                 double* t, double* u) {
    using DT = typename BlkDinv<MT>::T;
    const bool gv = !p.stage_vals;
    const int ld = 3 * p.R;
    const double w0 = poly_weight(p, 0);
    for (int e = threadIdx.x; e < NB * s.R; e += blockDim.x) {
        const int c = e / s.R, lr = e - c * s.R;
        const double* vc = v + (size_t)c * ld;
        double o0, o1, o2;
        blk_dinv<DT>(s.dinv, s.R, lr, p.omega, vc[3 * lr], vc[3 * lr + 1], vc[3 * lr + 2], o0, o1, o2);
        double* tc = t + (size_t)c * ld;
        double* zc = z + (size_t)c * ld;
        tc[3 * lr] = o0; tc[3 * lr + 1] = o1; tc[3 * lr + 2] = o2;
        zc[3 * lr] = w0 * o0; zc[3 * lr + 1] = w0 * o1; zc[3 * lr + 2] = w0 * o2;
    }
    __syncthreads();
    double* tc = t;
    double* tn = u;
    const int sub = threadIdx.x & 3;
    for (int k = 1; k < p.nterms; ++k) {
        const double wk = poly_weight(p, k);
        for (int lr0 = 0; lr0 < s.R; lr0 += blockDim.x / 4) {
            const int lr = lr0 + (threadIdx.x >> 2);
            double a[NB][3];
#pragma unroll
            for (int c = 0; c < NB; ++c) a[c][0] = a[c][1] = a[c][2] = 0.0;
            if (lr < s.R) {
                const int k1 = s.rp[lr + 1];
                for (int kk = s.rp[lr] + sub; kk < k1; kk += 4) {
                    const int ol = (int)s.lc[kk] - s.wown;
                    if (ol < 0 || ol >= s.R) continue;
                    const size_t o = kk, ps = s.pstride;
                    double b[9];
#pragma unroll
                    for (int e = 0; e < 9; ++e) b[e] = ldv(s, o + e * ps, gv);
#pragma unroll
                    for (int c = 0; c < NB; ++c) {
                        const double* xc = tc + (size_t)c * ld + 3 * ol;
                        const double x0 = xc[0], x1 = xc[1], x2 = xc[2];
                        a[c][0] += b[0] * x0 + b[1] * x1 + b[2] * x2;
                        a[c][1] += b[3] * x0 + b[4] * x1 + b[5] * x2;
                        a[c][2] += b[6] * x0 + b[7] * x1 + b[8] * x2;
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < NB; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    a[c][d] += __shfl_xor_sync(0xffffffffu, a[c][d], 1);
                    a[c][d] += __shfl_xor_sync(0xffffffffu, a[c][d], 2);
                }
            if (lr < s.R && sub == 0) {
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    const double* cc = tc + (size_t)c * ld + 3 * lr;
                    double y0 = a[c][0], y1 = a[c][1], y2 = a[c][2];
                    const double c0 = cc[0], c1 = cc[1], c2 = cc[2];
                    if (split) add_dact(p, s.rb + lr, c0, c1, c2, y0, y1, y2);
                    double e0, e1, e2;
                    blk_dinv<DT>(s.dinv, s.R, lr, p.omega, y0, y1, y2, e0, e1, e2);
                    double* nn = tn + (size_t)c * ld + 3 * lr;
                    double* zz = z + (size_t)c * ld + 3 * lr;
                    nn[0] = c0 - e0; nn[1] = c1 - e1; nn[2] = c2 - e2;
                    zz[0] += wk * nn[0]; zz[1] += wk * nn[1]; zz[2] += wk * nn[2];
                }
            }
        }
        __syncthreads();
        double* tmp = tc; tc = tn; tn = tmp;
    }
}

// ---------------------------------------------------------------------------
// Y = L V on each part (columns of the part's components), Y at the coupled
// dofs, the CTA's compact rows of V, and its partial of G = V^T Y (dense kmax^2)
// ---------------------------------------------------------------------------
template <class MT>
__global__ void __launch_bounds__(kThreads, 1) block_y_kernel(const BlockPlan p_arg) {
    __shared__ __align__(16) unsigned char s_p_raw[sizeof(BlockPlan)];
    BlockPlan& p = *reinterpret_cast<BlockPlan*>(s_p_raw);
    if (threadIdx.x == 0) p = p_arg;
    __syncthreads();
    extern __shared__ __align__(16) unsigned char sm[];
    const int cta = blockIdx.x;
    const Slice<MT> s = stage_slice<MT>(p, cta, sm);
    int* s_cols = reinterpret_cast<int*>(sm + p.off_cols);
    int* s_slot = s_cols + p.kmax;
    double* vec = reinterpret_cast<double*>(sm + p.off_vec);
    const int R3 = 3 * p.R;
    double* v = vec;                 // four regions of 4 columns x 3 R doubles
    double* z = vec + 4 * R3;
    double* t = vec + 8 * R3;
    double* u = vec + 12 * R3;
    int* s_act = reinterpret_cast<int*>(sm + p.off_act);
    for (int e = threadIdx.x; e < s.na; e += blockDim.x) s_act[e] = p.actp[s.ab + e] - 3 * s.rb;
    const int ncols = build_cols(p, cta, s_cols, s_slot);
    const int k = *p.rank;
    const bool split = p.dact != nullptr;
    // Y at the coupled dofs: zero the CTA's rows first (columns of other components stay zero)
    for (int e = threadIdx.x; e < s.na * p.kmax; e += blockDim.x) {
        const int j = e / s.na, il = e - j * s.na;
        p.Yact[(size_t)j * p.a + s.ab + il] = 0.0;
    }
    __syncthreads();
    constexpr int NB = 4;  // columns per pass over the blocks
    for (int q0 = 0; q0 < ncols; q0 += NB) {
        for (int e = threadIdx.x; e < NB * R3; e += blockDim.x) v[e] = 0.0;
        __syncthreads();
        for (int e = threadIdx.x; e < NB * s.na; e += blockDim.x) {
            const int c = e / s.na, il = e - c * s.na;
            if (q0 + c < ncols) v[(size_t)c * R3 + s_act[il]] = p.V[(size_t)s_cols[q0 + c] * p.a + p.actperm[s.ab + il]];
        }
        __syncthreads();
        local_poly_multi<MT, NB>(p, s, split, v, z, t, u);
        for (int e = threadIdx.x; e < NB * s.R; e += blockDim.x) {
            const int c = e / s.R, lr = e - c * s.R;
            if (q0 + c >= ncols) continue;
            const double* zc = z + (size_t)c * R3 + 3 * lr;
            float* Yj = p.Y + (size_t)s_cols[q0 + c] * 4 * p.n;
            reinterpret_cast<float4*>(Yj)[s.rb + lr] = make_float4((float)zc[0], (float)zc[1], (float)zc[2], 0.f);
        }
        // the PCG applies the FP32 copy of Y; the Woodbury core is built from the same rounded values
        for (int e = threadIdx.x; e < NB * s.na; e += blockDim.x) {
            const int c = e / s.na, il = e - c * s.na;
            if (q0 + c < ncols)
                p.Yact[(size_t)s_cols[q0 + c] * p.a + s.ab + il] = (double)(float)z[(size_t)c * R3 + s_act[il]];
        }
        __syncthreads();
    }
    // the CTA's coupled rows of V, compact: [list position q][own coupled dof]
    {
        double* Vc = p.Vc + (size_t)p.kmax * s.ab;
        for (int e = threadIdx.x; e < ncols * s.na; e += blockDim.x) {
            const int q = e / s.na, il = e - q * s.na;
            Vc[e] = p.V[(size_t)s_cols[q] * p.a + p.actperm[s.ab + il]];
        }
    }
    // partial G_c[j][l] = sum_{own coupled dofs} V[., j] Yact[., l]  (dense kmax^2, zero outside).
    // The CTA's rows of V ([q][dof]) and of Y ([dof][q]) are staged in the (now free) vector region
    // when they fit: a warp takes a row q_a, its lanes the columns q_b, and walks the dofs.
    const int aidx = p.cta_aidx[cta];
    if (aidx >= 0) {  // uniform in the CTA
        __syncthreads();  // the compact rows of V above are read back below
        double* Gc = p.pG + (size_t)aidx * p.kmax * p.kmax;
        for (int e = threadIdx.x; e < p.kmax * p.kmax; e += blockDim.x) Gc[e] = 0.0;
        const bool staged = 2 * (size_t)s.na * ncols <= (size_t)16 * R3;
        double* Vs = vec;
        double* Ys = vec + (size_t)s.na * ncols;
        if (staged)
            for (int e = threadIdx.x; e < ncols * s.na; e += blockDim.x) {
                const int q = e / s.na, il = e - q * s.na;
                Vs[e] = p.Vc[(size_t)p.kmax * s.ab + e];
                Ys[(size_t)il * ncols + q] = p.Yact[(size_t)s_cols[q] * p.a + s.ab + il];
            }
        __syncthreads();
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int qa = warp; qa < ncols; qa += kWarps)
            for (int qb = lane; qb < ncols; qb += 32) {
                const int j = s_cols[qa], l = s_cols[qb];
                double acc = 0.0;
                if (staged) {
                    for (int il = 0; il < s.na; ++il) acc += Vs[(size_t)qa * s.na + il] * Ys[(size_t)il * ncols + qb];
                } else {
                    for (int il = 0; il < s.na; ++il)
                        acc += p.Vc[(size_t)p.kmax * s.ab + (size_t)qa * s.na + il] * p.Yact[(size_t)l * p.a + s.ab + il];
                }
                if (j < k && l < k) Gc[(size_t)j * p.kmax + l] = acc;
            }
    }
}

// G[e] = sum over the coupled CTAs of their partials (fixed order), symmetrised later
__global__ void block_g_reduce_kernel(const double* pG, int nact, int kk, double* G) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kk) return;
    double acc = 0.0;
    for (int c = 0; c < nact; ++c) acc += pG[(size_t)c * kk + e];
    G[e] = acc;
}

// Kinv = diag(1/d) - sym(T) over the leading k x k (identity beyond k)
__global__ void block_kinv_kernel(const double* T, const double* d, const int* dk, int kmax, double* Kinv) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kmax * kmax) return;
    const int i = e / kmax, j = e - i * kmax;
    const int k = *dk;
    double v;
    if (i < k && j < k) v = (i == j ? 1.0 / d[i] : 0.0) - 0.5 * (T[e] + T[(size_t)j * kmax + i]);
    else v = (i == j) ? 1.0 : 0.0;
    Kinv[e] = v;
}

// K = 0 when K^-1 was not SPD (the preconditioner falls back to L alone); symmetrise otherwise
__global__ void block_k_finish_kernel(double* K, int kmax, const int* dk, const int* bad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kmax * kmax) return;
    const int i = e / kmax, j = e - i * kmax;
    if (*bad || i >= *dk || j >= *dk) { K[e] = 0.0; return; }
    if (j < i) {
        const double a = K[e], b = K[(size_t)j * kmax + i];
        K[e] = 0.5 * (a + b);
        K[(size_t)j * kmax + i] = 0.5 * (a + b);
    }
}

// ---------------------------------------------------------------------------
// the pipelined PCG.  Per pass, with v the vector the preconditioner takes
// (r on a (re)start, w otherwise):
//   phase 1: mt = L v (local), partials of Y^T v and of the dots (r,u) (w,u) (r,r)
//   -- grid barrier --
//   phase 2: s = Y^T v, c = K s on the CTA's columns, m = mt + Y c (published),
//            partials of V^T m; dots summed -> stop test, alpha, beta
//   -- grid barrier --
//   phase 3: window of m, vt = V^T m, n = D m - V C vt, then either
//            (u, w) = (m, n) on a (re)start, or the recurrences
//            z = n + b z, q = m + b q, s = w + b s, p = u + b p,
//            x += a p, r -= a s, u -= a q, w -= a z
// A true-residual check (r = rhs - S x, two more barriers) runs when the
// recursive residual reaches tol, at max_iter, and every rr_every iterations;
// if it fails the PCG restarts from the true residual.  Every CTA sums the same
// partials in the same order, so all CTAs take the same decisions.
// ---------------------------------------------------------------------------
enum { kPassStart = 0, kPassNormal = 1 };

template <class MT>
__global__ void __launch_bounds__(kThreads, 1) block_pcg_kernel(const BlockPlan p_arg) {
    __shared__ __align__(16) unsigned char s_p_raw[sizeof(BlockPlan)];
    BlockPlan& p = *reinterpret_cast<BlockPlan*>(s_p_raw);
    if (threadIdx.x == 0) p = p_arg;
    __syncthreads();
    extern __shared__ __align__(16) unsigned char sm[];
    const int cta = blockIdx.x;
    const unsigned int G = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Slice<MT> sl = stage_slice<MT>(p, cta, sm);
    const bool gv = !p.stage_vals;
    const bool split = p.dact != nullptr;
    const int R = sl.R, R3 = 3 * R, ld = 3 * p.R;
    double* vec = reinterpret_cast<double*>(sm + p.off_vec);
    double* X = vec;             // own-row vectors, 3 per row
    double* Rr = vec + ld;
    double* Uu = vec + 2 * ld;
    double* Ww = vec + 3 * ld;
    double* Pp = vec + 4 * ld;
    double* Ss = vec + 5 * ld;
    double* Qq = vec + 6 * ld;
    double* Zz = vec + 7 * ld;
    double* Mm = vec + 8 * ld;
    double* Mt = vec + 9 * ld;
    double* T0 = vec + 10 * ld;
    double* T1 = vec + 11 * ld;
    double* Nn = T0;             // n = S m (phase 3) reuses the polynomial's scratch (phase 1)
    double* win = reinterpret_cast<double*>(sm + p.off_win);   // 4 per window node
    int* s_act = reinterpret_cast<int*>(sm + p.off_act);       // own coupled dofs, local (3 lr + d)
    int* s_cols = reinterpret_cast<int*>(sm + p.off_cols);
    int* s_slot = s_cols + p.kmax;
    double* s_sv = reinterpret_cast<double*>(sm + p.off_kv);  // Y^T v sums (kmax)
    double* s_vt = s_sv + p.kmax;                             // V^T m sums (kmax)
    double* s_c = s_vt + p.kmax;                              // K s on the CTA's columns (by list position)
    double* s_t = s_c + p.kmax;                               // C vt on the CTA's columns
    double* s_red = reinterpret_cast<double*>(sm + p.off_red);// kWarps x 4 scratch
    __shared__ double s_dot[4];
    __shared__ int s_ok;
    for (int e = threadIdx.x; e < sl.na; e += blockDim.x) s_act[e] = p.actp[sl.ab + e] - 3 * sl.rb;
    const int ncols = build_cols(p, cta, s_cols, s_slot);
    const int k = *p.rank;
    int epoch = 0;
    const bool yc_on = p.stage_yc && ncols <= p.NCOL;
    if (yc_on) {
        float* yc = reinterpret_cast<float*>(sm + p.off_yc);
        for (int e = threadIdx.x; e < ncols * R; e += blockDim.x) {
            const int q = e / R, lr = e - q * R;
            const float4 y = reinterpret_cast<const float4*>(p.Y + (size_t)s_cols[q] * 4 * p.n)[sl.rb + lr];
            float* o = yc + (size_t)q * ld + 3 * lr;
            o[0] = y.x; o[1] = y.y; o[2] = y.z;
        }
        __syncthreads();
    }

    // grid barrier: the CTA's partials are already in global memory
    auto barrier = [&]() -> bool {
        __syncthreads();
        if (threadIdx.x == 0) s_ok = grid_arrive_wait(p.bar, G, p.spin_limit, epoch);
        ++epoch;
        __syncthreads();
        return s_ok != 0;
    };
    // CTA sums of per-thread values -> pdot[cta * 4 + i] for i in [i0, i1).  The pass's dots use
    // slots 0-2 and the true-residual check slot 3: a check's slot is still being read when a fast
    // CTA already writes the next pass's dots (no barrier between the two)
    auto cta_partials = [&](double a0, double a1, double a2, double a3, double* out, int i0, int i1) {
        a0 = bwarp_sum(a0); a1 = bwarp_sum(a1); a2 = bwarp_sum(a2); a3 = bwarp_sum(a3);
        if (lane == 0) { s_red[4 * warp] = a0; s_red[4 * warp + 1] = a1; s_red[4 * warp + 2] = a2; s_red[4 * warp + 3] = a3; }
        __syncthreads();
        if ((int)threadIdx.x >= i0 && (int)threadIdx.x < i1) {
            double t = 0.0;
            for (int w = 0; w < kWarps; ++w) t += s_red[4 * w + threadIdx.x];
            out[4 * cta + threadIdx.x] = t;
        }
    };
    // the dots of all CTAs, summed in CTA order by warp 0 (same bits everywhere)
    auto sum_dots = [&]() {
        if (warp == 0) {
            double a[4] = {0, 0, 0, 0};
            for (unsigned c = lane; c < G; c += 32)
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] += p.pdot[4 * c + i];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = bwarp_sum(a[i]);
            if (lane == 0)
#pragma unroll
                for (int i = 0; i < 4; ++i) s_dot[i] = a[i];
        }
    };
    // out[j] = sum of the contributor slots of column j's component, for every j < k; each warp
    // issues the loads of four columns before it reduces them (one round trip serves four)
    auto sum_slots = [&](const double* part, double* out) {
        for (int j0 = 4 * warp; j0 < k; j0 += 4 * kWarps) {
            double a[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = 0.0;
                const int j = j0 + u;
                if (j < k) {
                    const int g = p.comp_of_col[j];
                    if (g >= 0)
                        for (int q = p.comp_slot_ptr[g] + lane; q < p.comp_slot_ptr[g + 1]; q += 32)
                            a[u] += part[(size_t)q * p.kmax + j];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double t = bwarp_sum(a[u]);
                if (lane == 0 && j0 + u < k) out[j0 + u] = t;
            }
        }
    };
    // the CTA's Y columns at its own rows: shared memory (FP32) when staged
    const float* Yc = yc_on ? reinterpret_cast<const float*>(sm + p.off_yc) : nullptr;
    auto yval = [&](int q, int lr, int d) -> double {
        if (Yc) return (double)Yc[(size_t)q * ld + 3 * lr + d];
        const float* yj = p.Y + (size_t)s_cols[q] * 4 * p.n + 4 * (size_t)(sl.rb + lr);
        return (double)__ldg(yj + d);
    };
    // partials of Y^T v over the own rows -> part[slot][j] for the CTA's columns
    auto y_partials = [&](const double* v, double* part) {
        for (int q = warp; q < ncols; q += kWarps) {
            double a = 0.0;
            for (int lr = lane; lr < R; lr += 32)
                a += yval(q, lr, 0) * v[3 * lr] + yval(q, lr, 1) * v[3 * lr + 1] + yval(q, lr, 2) * v[3 * lr + 2];
            a = bwarp_sum(a);
            if (lane == 0) part[(size_t)s_slot[q] * p.kmax + s_cols[q]] = a;
        }
    };
    // the CTA's coupled rows of V, compact ([list position][own coupled dof], written by the Y kernel)
    const double* Vc = p.Vc + (size_t)p.kmax * sl.ab;
    // partials of V^T v over the own coupled dofs
    auto v_partials = [&](const double* v, double* part) {
        if (sl.na == 0) return;
        for (int q = warp; q < ncols; q += kWarps) {
            const double* vq = Vc + (size_t)q * sl.na;
            double a = 0.0;
            for (int il = lane; il < sl.na; il += 32) a += vq[il] * v[s_act[il]];
            a = bwarp_sum(a);
            if (lane == 0) part[(size_t)s_slot[q] * p.kmax + s_cols[q]] = a;
        }
    };
    // s_t[q] = (C vt)_j for the CTA's columns, then out[own coupled dof] -= (V C vt)
    auto lowrank_sub = [&](double* out) {
        if (sl.na == 0) return;
        for (int q = warp; q < ncols; q += kWarps) {
            const int j = s_cols[q];
            double a = 0.0;
            for (int l = lane; l < k; l += 32) a += p.C[(size_t)j * p.kmax + l] * s_vt[l];
            a = bwarp_sum(a);
            if (lane == 0) s_t[q] = a;
        }
        __syncthreads();
        for (int il = threadIdx.x; il < sl.na; il += blockDim.x) {
            double a = 0.0;
            int q = 0;
            for (; q + 8 <= ncols; q += 8) {
                double vv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) vv[u] = Vc[(size_t)(q + u) * sl.na + il];
#pragma unroll
                for (int u = 0; u < 8; ++u) a += vv[u] * s_t[q + u];
            }
            for (; q < ncols; ++q) a += Vc[(size_t)q * sl.na + il] * s_t[q];
            out[s_act[il]] -= a;
        }
    };
    // stage the window of a published vector (own rows from shared memory)
    auto stage = [&](const double* pub, const double* own) {
        for (int e = threadIdx.x; e < sl.nwin; e += blockDim.x) {
            const int node = sl.wn[e];
            double a0, a1, a2;
            if (node >= sl.rb && node < sl.re) {
                const double* o = own + 3 * (node - sl.rb);
                a0 = o[0]; a1 = o[1]; a2 = o[2];
            } else {
                Vec4<double>::load(pub, node, a0, a1, a2);
            }
            win[4 * e] = a0; win[4 * e + 1] = a1; win[4 * e + 2] = a2;
        }
    };
    // out = D v over the own rows (window staged), FP64 coupled diagonal blocks in the mixed modes
    auto op_spmv = [&](const double* vown, double* out) {
        auto epi = [&](int lr, double y0, double y1, double y2) {
            if (split) add_dact(p, sl.rb + lr, vown[3 * lr], vown[3 * lr + 1], vown[3 * lr + 2], y0, y1, y2);
            out[3 * lr] = y0; out[3 * lr + 1] = y1; out[3 * lr + 2] = y2;
        };
        slice_spmv<MT>(sl, gv, false, nullptr, win, epi);
    };

    // ---- prologue: x = 0, r = rhs ----
    for (int e = threadIdx.x; e < R; e += blockDim.x) {
        double r0, r1, r2;
        Vec4<double>::load(p.rhs, sl.rb + e, r0, r1, r2);
        Rr[3 * e] = r0; Rr[3 * e + 1] = r1; Rr[3 * e + 2] = r2;
        for (int d = 0; d < 3; ++d) {
            X[3 * e + d] = 0.0; Pp[3 * e + d] = 0.0; Ss[3 * e + d] = 0.0; Qq[3 * e + d] = 0.0; Zz[3 * e + d] = 0.0;
        }
    }
    __syncthreads();

    int pass = kPassStart, it = 0, status = -1, restarts = 0, npass = 0;
    // phase clocks (trace mode): 0 pass top, 1 polynomial done, 2 partials written, 3 after barrier A,
    // 4 sums read, 5 K s done, 6 m formed, 7 V^T m partials / decisions, 8 after barrier B, 9 window
    // staged, 10 V^T m summed, 11 D m done, 12 low-rank done, 13 updates done
    auto mark = [&](int ev) {
        if (p.trace && threadIdx.x == 0 && npass < p.trace_iters)
            p.trace[((size_t)cta * p.trace_iters + npass) * 16 + ev] = (unsigned long long)clock64();
    };
    double normb = -1.0, rel = 1.0, alpha = 0.0, beta = 0.0, alpha_prev = 0.0, gamma_prev = 0.0;
    bool fresh = true;  // next normal pass is the first after a (re)start: beta = 0
    for (;;) {
        // ---------------- phase 1 ----------------
        mark(0);
        const double* v = pass == kPassStart ? Rr : Ww;
        local_poly<MT>(p, sl, split, v, Mt, T0, T1);
        mark(1);
        y_partials(v, p.pY);
        {
            double g = 0, d = 0, rr = 0;
            for (int e = threadIdx.x; e < R3; e += blockDim.x) {
                const double r = Rr[e];
                rr += r * r;
                if (pass == kPassNormal) { g += r * Uu[e]; d += Ww[e] * Uu[e]; }
            }
            cta_partials(g, d, rr, 0.0, p.pdot, 0, 3);
        }
        mark(2);
        if (!barrier()) return;
        mark(3);
        // ---------------- phase 2 ----------------
        sum_slots(p.pY, s_sv);
        sum_dots();
        __syncthreads();
        mark(4);
        for (int q = warp; q < ncols; q += kWarps) {
            const int j = s_cols[q];
            double a = 0.0;
            for (int l = lane; l < k; l += 32) a += p.K[(size_t)j * p.kmax + l] * s_sv[l];
            a = bwarp_sum(a);
            if (lane == 0) s_c[q] = a;
        }
        __syncthreads();
        mark(5);
        for (int e = threadIdx.x; e < R; e += blockDim.x) {
            double m0 = Mt[3 * e], m1 = Mt[3 * e + 1], m2 = Mt[3 * e + 2];
            for (int q = 0; q < ncols; ++q) {
                const double c = s_c[q];
                m0 += yval(q, e, 0) * c; m1 += yval(q, e, 1) * c; m2 += yval(q, e, 2) * c;
            }
            Mm[3 * e] = m0; Mm[3 * e + 1] = m1; Mm[3 * e + 2] = m2;
            Vec4<double>::store(p.mpub, sl.rb + e, m0, m1, m2);
        }
        __syncthreads();
        mark(6);
        v_partials(Mm, p.pV);
        // decisions (identical in every CTA)
        bool check = false;
        {
            const double gam = s_dot[0], del = s_dot[1], rr = s_dot[2];
            if (normb < 0) {
                normb = sqrt(rr);
                if (!(normb > 0)) status = isfinite(normb) ? 0 : 3;
                rel = normb > 0 ? 1.0 : 0.0;
            }
            if (status < 0 && pass == kPassNormal) {
                rel = sqrt(rr) / normb;
                if (!isfinite(rel)) status = 3;
                else if (rel <= p.tol || it >= p.max_iter || (p.rr_every > 0 && it > 0 && it % p.rr_every == 0 && !fresh))
                    check = true;
                else {
                    beta = fresh ? 0.0 : gam / gamma_prev;
                    const double den = fresh ? del : del - beta * gam / alpha_prev;
                    if (!(isfinite(den) && den > 0 && isfinite(gam) && gam > 0)) status = 3;
                    else {
                        alpha = gam / den;
                        if (cta == 0 && threadIdx.x == 0 && it < p.max_coef) {
                            p.cg_coef[2 * it] = alpha;
                            if (it > 0) p.cg_coef[2 * (it - 1) + 1] = beta;
                        }
                        alpha_prev = alpha;
                        gamma_prev = gam;
                    }
                }
            }
        }
        if (status >= 0) break;
        mark(7);
        if (!barrier()) return;
        mark(8);
        // ---------------- phase 3 ----------------
        if (!check) {
            stage(p.mpub, Mm);
            __syncthreads();
            mark(9);
            sum_slots(p.pV, s_vt);
            __syncthreads();
            mark(10);
            op_spmv(Mm, Nn);
            __syncthreads();
            mark(11);
            lowrank_sub(Nn);
            __syncthreads();
            mark(12);
            if (pass == kPassStart) {
                for (int e = threadIdx.x; e < R3; e += blockDim.x) { Uu[e] = Mm[e]; Ww[e] = Nn[e]; }
                pass = kPassNormal;
                fresh = true;
            } else {
                for (int e = threadIdx.x; e < R3; e += blockDim.x) {
                    const double z = Nn[e] + beta * Zz[e], q = Mm[e] + beta * Qq[e];
                    const double sv = Ww[e] + beta * Ss[e], pv = Uu[e] + beta * Pp[e];
                    Zz[e] = z; Qq[e] = q; Ss[e] = sv; Pp[e] = pv;
                    X[e] += alpha * pv;
                    Rr[e] -= alpha * sv;
                    Uu[e] -= alpha * q;
                    Ww[e] -= alpha * z;
                }
                ++it;
                fresh = false;
            }
            __syncthreads();
            mark(13);
            ++npass;
            continue;
        }
        // ---------------- true residual: r = rhs - (D x - V C V^T x) ----------------
        for (int e = threadIdx.x; e < R; e += blockDim.x)
            Vec4<double>::store(p.xpub, sl.rb + e, X[3 * e], X[3 * e + 1], X[3 * e + 2]);
        __syncthreads();
        v_partials(X, p.pX);
        if (!barrier()) return;
        stage(p.xpub, X);
        sum_slots(p.pX, s_vt);
        __syncthreads();
        op_spmv(X, Nn);
        __syncthreads();
        lowrank_sub(Nn);
        __syncthreads();
        {
            double rr = 0.0;
            for (int e = threadIdx.x; e < R; e += blockDim.x) {
                double b0, b1, b2;
                Vec4<double>::load(p.rhs, sl.rb + e, b0, b1, b2);
                const double r0 = b0 - Nn[3 * e], r1 = b1 - Nn[3 * e + 1], r2 = b2 - Nn[3 * e + 2];
                Rr[3 * e] = r0; Rr[3 * e + 1] = r1; Rr[3 * e + 2] = r2;
                rr += r0 * r0 + r1 * r1 + r2 * r2;
            }
            cta_partials(0.0, 0.0, 0.0, rr, p.pdot, 3, 4);
        }
        if (!barrier()) return;
        sum_dots();
        __syncthreads();
        rel = sqrt(s_dot[3]) / normb;
        ++restarts;
        if (rel <= p.tol) { status = 0; break; }
        if (it >= p.max_iter) { status = 4; break; }
        if (!isfinite(rel)) { status = 3; break; }
        pass = kPassStart;  // restart from the true residual
    }
    // ---- x out (own rows) and the scalars ----
    for (int e = threadIdx.x; e < R; e += blockDim.x) Vec4<double>::store(p.x, sl.rb + e, X[3 * e], X[3 * e + 1], X[3 * e + 2]);
    if (cta == 0 && threadIdx.x == 0) {
        p.out[0] = it; p.out[1] = rel; p.out[2] = status; p.out[3] = normb; p.out[4] = restarts;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_block_columns(const BlockPlan& p, cudaStream_t st) {
    count_launch();
    block_columns_kernel<<<1, 256, 0, st>>>(p);
}

template <class MT>
static cudaError_t launch_y_t(const BlockPlan& p, cudaStream_t st) {
    auto fn = block_y_kernel<MT>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_y);
    if (e != cudaSuccess) return e;
    count_launch();
    fn<<<p.G_ctas, kThreads, p.smem_y, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_block_y(int precision, const BlockPlan& p, cudaStream_t st) {
    return precision == 0 ? launch_y_t<double>(p, st) : launch_y_t<float>(p, st);
}

void launch_block_k(const BlockPlan& p, int nact_cta, cudaStream_t st) {
    const int kk = p.kmax * p.kmax;
    const int* dk = p.rank;
    count_launch();
    block_g_reduce_kernel<<<(kk + 255) / 256, 256, 0, st>>>(p.pG, nact_cta, kk, p.G);
    // Ka = G Lc, Kb = Lc^T Ka
    GemmArgs g1{p.G, p.Lc, p.Ka, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 0, 0, 1.0, 0.0};
    launch_gemm(g1, p.kmax, p.kmax, st);
    GemmArgs g2{p.Lc, p.Ka, p.Kb, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 1, 0, 1.0, 0.0};
    launch_gemm(g2, p.kmax, p.kmax, st);
    count_launch();
    block_kinv_kernel<<<(kk + 255) / 256, 256, 0, st>>>(p.Kb, p.dpiv, dk, p.kmax, p.Ka);
    // K~ = (K^-1)^-1 into Kb (Cholesky: flags a matrix that is not SPD)
    cudaMemsetAsync(p.bad, 0, sizeof(int), st);
    if (!launch_chol_inverse(p.Ka, p.kmax, p.Kb, p.bad, st)) {
        launch_cholesky(p.Ka, p.kmax, p.G, p.bad, st);
        launch_chol_solve(p.G, p.kmax, p.ident, p.kmax, p.Kb, p.kmax, p.kmax, nullptr, p.pG, st);
    }
    // K = Lc K~ Lc^T
    GemmArgs g3{p.Lc, p.Kb, p.Ka, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 0, 0, 1.0, 0.0};
    launch_gemm(g3, p.kmax, p.kmax, st);
    GemmArgs g4{p.Ka, p.Lc, p.K, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 0, 1, 1.0, 0.0};
    launch_gemm(g4, p.kmax, p.kmax, st);
    count_launch();
    block_k_finish_kernel<<<(kk + 255) / 256, 256, 0, st>>>(p.K, p.kmax, dk, p.bad);
}

template <class MT>
static cudaError_t launch_pcg_t(const BlockPlan& p, cudaStream_t st) {
    auto fn = block_pcg_kernel<MT>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, p.smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm < 1 || p.G_ctas > per_sm * sms) return cudaErrorCooperativeLaunchTooLarge;
    BlockPlan arg = p;
    void* args[] = {&arg};
    count_launch();
    return cudaLaunchCooperativeKernel((void*)fn, dim3(p.G_ctas), dim3(kThreads), args, p.smem, st);
}

cudaError_t launch_block_pcg(int precision, const BlockPlan& p, cudaStream_t st) {
    return precision == 0 ? launch_pcg_t<double>(p, st) : launch_pcg_t<float>(p, st);
}

int block_max_smem() { return 227 * 1024 - 4096; }

// shared-memory layouts for the maxima in p (R, BLK, W, NA, NCOL, kmax): a common prefix (row
// pointers, window positions, Dd^-1, window, coupled dofs, column lists, k-vectors, the value planes),
// then the vectors: 16 x 3R doubles in the Y kernel (four regions of four), 12 x 3R in the PCG followed
// by the CTA's Y columns (FP32)
size_t block_smem_bytes(int precision, BlockPlan& p, bool stage_vals, bool stage_yc) {
    const size_t mt = precision == 0 ? 8 : 4, dt = precision == 0 ? 8 : 4;
    auto al = [](size_t b) { return (b + 15) / 16 * 16; };
    size_t off = 0;
    p.off_rp = (int)off; off += al(sizeof(int) * (p.R + 1));
    p.off_lc = (int)off; off += al(sizeof(unsigned short) * p.BLK);
    p.off_dinv = (int)off; off += al(dt * 9 * p.R);
    p.off_wn = (int)off; off += al(sizeof(int) * p.W);
    p.off_win = (int)off; off += al(sizeof(double) * 4 * p.W);
    p.off_act = (int)off; off += al(sizeof(int) * p.NA);
    p.off_cols = (int)off; off += al(sizeof(int) * 2 * p.kmax);
    p.off_kv = (int)off; off += al(sizeof(double) * 4 * p.kmax);
    p.off_red = (int)off; off += al(sizeof(double) * 4 * kWarps);
    p.off_val = (int)off;
    p.stage_vals = stage_vals ? 1 : 0;
    if (stage_vals) off += al(mt * 9 * p.BLK);
    p.off_vec = (int)off;
    p.smem_y = off + al(sizeof(double) * 16 * 3 * (size_t)p.R);
    off += al(sizeof(double) * 12 * 3 * (size_t)p.R);
    p.off_yc = (int)off;
    p.stage_yc = stage_yc ? 1 : 0;
    if (stage_yc) off += al(sizeof(float) * 3 * (size_t)p.R * p.NCOL);
    p.smem = off;
    return std::max(p.smem, p.smem_y);
}

}  // namespace hsc
