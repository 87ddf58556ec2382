// Persistent Schur-complement PCG for one or many HSC systems.
//
// One cooperative launch (one 512-thread CTA per SM) runs the whole PCG loop
// of linear_hsc.cu:359-393 (core.py:95-138 is the oracle's form) for every
// system of a batch.  Each CTA owns a contiguous range of FEM block rows of
// one system; grid-wide barriers with bounded waits separate the phases:
//
//   A  p = z + beta p_prev (formed on the fly in the gathers),  y = D p,
//      tt_j = (Vt^T z)_j + beta tt_j by designated warps (the Vt^T z
//      partials were produced per CTA at the end of the previous phase),
//      partial p.Dp - sum_j d_j tt_j^2
//   -- barrier --
//   B  alpha = rz / pSp;  y[act] -= Vt (d .* tt);  x += alpha p;
//      r -= alpha y;  t = w Dd^-1 r;  z = w_0 t;  partial r.r
//   -- barrier --
//   C_k (k = 1 .. terms-1): t' = t - w Dd^-1 (D t);  z += w_k t';
//      partial r.z and the CTA's Vt^T z partials after the last term
//   -- barrier each --
//
// With the Schur basis (the learned polynomial) the terms run on S instead of
// D: t' = t - w Dd^-1 (D t - Vt d Vt^T t).  Every phase that writes a term
// also leaves the CTA's partials of Vt^T t (ping-pong by term parity), and
// the next C phase sums them before its SpMV and subtracts the low-rank part
// at its coupled rows; the barrier count stays the same.
//
// so one iteration costs terms+1 barriers and `terms` passes over D.  All
// scalars are reduced redundantly, in the same order, by every CTA of a
// system: no floating-point atomics, bit-reproducible results.  The true
// residual check at convergence (linear_hsc.cu:375-387) and the FP64 residual
// replacement of the mixed-precision modes run as a replacement slot
// (A' r = rhs - D x in FP64, B' r += Vt d Vt^T x) with the same barrier count.
//
// On a vehicle-size system the ~20 MB matrix stays in L2 and one iteration is
// bound by latency, so the kernel shortens dependent chains: the CTA partial
// is folded into the barrier arrival (release add, acquire poll), the r.r and
// r.z partials are fetched in one pass, the SpMV issues the column indices and
// gathers of several blocks before using them, and each CTA keeps its block of
// Vt (the rows of its own coupled dofs) in shared memory for the whole solve.
#include "../../include/hsc_c_api.h"
#include <type_traits>

#include "hsc_check.cuh"
#include "hsc_internal.cuh"

namespace hsc {

namespace {

template <class MT> struct Cmp { using T = float; };
template <> struct Cmp<double> { using T = double; };
template <class MT> struct DinvT { using T = float; };
template <> struct DinvT<double> { using T = double; };

// b0 x0 + b1 x1 + b2 x2 with explicit fused multiply-adds, so the rounding
// does not depend on how the compiler contracts the surrounding code
__device__ __forceinline__ float dot3(float b0, float b1, float b2, float x0, float x1, float x2) {
    return __fmaf_rn(b2, x2, __fmaf_rn(b1, x1, b0 * x0));
}
__device__ __forceinline__ double dot3(double b0, double b1, double b2, double x0, double x1, double x2) {
    return __fma_rn(b2, x2, __fma_rn(b1, x1, b0 * x0));
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class VT>
__device__ __forceinline__ VT& elem(void* v, int dof) {
    return reinterpret_cast<VT*>(v)[4 * (dof / 3) + dof % 3];
}

// warp-level sums of a[b..e) and (optionally) c[b..e), loads issued before the
// adds, fixed order: the same bits in every CTA.  Valid in lane 0.
__device__ __forceinline__ void warp_sum_parts(const double* pa, const double* pc, int b, int e, double& sa,
                                               double& sc) {
    const int lane = threadIdx.x & 31;
    double va[8], vc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = b + lane + 32 * q;
        va[q] = i < e ? pa[i] : 0.0;
        vc[q] = (pc && i < e) ? pc[i] : 0.0;
    }
    sa = 0.0;
    sc = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) { sa += va[q]; sc += vc[q]; }
    for (int i = b + lane + 256; i < e; i += 32) {
        sa += pa[i];
        if (pc) sc += pc[i];
    }
    sa = warp_sum(sa);
    sc = warp_sum(sc);
}

// y_row = sum_k B_k x[col_k] over the rows this warp owns (a contiguous,
// block-balanced range).  Lanes walk the warp's consecutive blocks, so the 9
// value planes are read coalesced; the products are summed per row by a
// shuffle segmented scan (rows are nondecreasing along the blocks), and the
// tail lane of each row segment adds its sum into s_y: one writer per row and
// slice, slices in order, so the result is deterministic.  Then each lane runs
// the epilogue of one owned row.
//
// The warp loads NB slices of 32 blocks (indices, gathers and values) before
// it scans the first one, so one round trip to L2 serves NB slices: the loop
// is bound by load latency, not bandwidth, on an L2-resident matrix.
template <int NB, class MT, class CT, class Gather, class Epi>
__device__ __forceinline__ void spmv_warp(int wr0, int wr1, int rb, const int* __restrict__ rowptr,
                                          const int* __restrict__ colidx, const int* __restrict__ rowid,
                                          const int* s_col, const int* s_row, int kcta0, const MT* __restrict__ vals,
                                          int nnz, double* s_y, const Gather& gather, Epi& epi) {
    const int lane = threadIdx.x & 31;
    if (wr1 <= wr0) return;
    const int k0 = __ldg(rowptr + wr0), k1 = __ldg(rowptr + wr1);
    for (int r = wr0 + lane; r < wr1; r += 32) {
        double* yy = s_y + 3 * (r - rb);
        yy[0] = 0.0; yy[1] = 0.0; yy[2] = 0.0;
    }
    __syncwarp();
    const size_t st = (size_t)nnz;
    for (int kb = k0; kb < k1; kb += 32 * NB) {
        CT p0[NB], p1[NB], p2[NB];
        int row[NB];
#pragma unroll
        for (int h = 0; h < NB; ++h) {
            const int k = kb + 32 * h + lane;
            const bool valid = k < k1;
            int c = 0;
            row[h] = -1;
            if (valid) {
                if (s_col) { c = s_col[k - kcta0]; row[h] = s_row[k - kcta0]; }
                else { c = __ldg(colidx + k); row[h] = __ldg(rowid + k); }
            }
            p0[h] = 0; p1[h] = 0; p2[h] = 0;
            if (valid) {
                CT x0, x1, x2;
                gather(c, x0, x1, x2);
                const MT* v = vals + k;
                const CT b0 = Num<MT>::get(__ldg(v)), b1 = Num<MT>::get(__ldg(v + st)),
                         b2 = Num<MT>::get(__ldg(v + 2 * st)), b3 = Num<MT>::get(__ldg(v + 3 * st)),
                         b4 = Num<MT>::get(__ldg(v + 4 * st)), b5 = Num<MT>::get(__ldg(v + 5 * st)),
                         b6 = Num<MT>::get(__ldg(v + 6 * st)), b7 = Num<MT>::get(__ldg(v + 7 * st)),
                         b8 = Num<MT>::get(__ldg(v + 8 * st));
                p0[h] = dot3(b0, b1, b2, x0, x1, x2);
                p1[h] = dot3(b3, b4, b5, x0, x1, x2);
                p2[h] = dot3(b6, b7, b8, x0, x1, x2);
            }
        }
#pragma unroll
        for (int h = 0; h < NB; ++h) {
            CT a0 = p0[h], a1 = p1[h], a2 = p2[h];
            const int rw = row[h];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int rr = __shfl_up_sync(0xffffffffu, rw, off);
                const CT q0 = __shfl_up_sync(0xffffffffu, a0, off);
                const CT q1 = __shfl_up_sync(0xffffffffu, a1, off);
                const CT q2 = __shfl_up_sync(0xffffffffu, a2, off);
                if (lane >= off && rr == rw) { a0 += q0; a1 += q1; a2 += q2; }
            }
            const int rn = __shfl_down_sync(0xffffffffu, rw, 1);
            if (rw >= 0 && (lane == 31 || rn != rw)) {
                double* yy = s_y + 3 * (rw - rb);
                yy[0] += (double)a0; yy[1] += (double)a1; yy[2] += (double)a2;
            }
            __syncwarp();
        }
    }
    __syncwarp();
    for (int r = wr0 + lane; r < wr1; r += 32) {
        const double* yy = s_y + 3 * (r - rb);
        epi(r, (CT)yy[0], (CT)yy[1], (CT)yy[2]);
    }
}

// spmv_warp over the CTA's shared-memory copy: value planes s_val[e * nblk +
// kl], window positions of the columns (s_lc) and local rows (s_lr) of the
// CTA's blocks, and the staged vector window s_win (4 entries per node).
// Same slices, scan and summation order as spmv_warp.
template <int NB, class MT, class CT, class VT, class Epi>
__device__ __forceinline__ void spmv_warp_res(int wr0, int wr1, int rb, const int* __restrict__ rowptr, int kcta0,
                                              int nblk, const MT* s_val, const unsigned short* s_lc,
                                              const unsigned short* s_lr, const VT* s_win, double* s_y, Epi& epi) {
    const int lane = threadIdx.x & 31;
    if (wr1 <= wr0) return;
    const int k0 = __ldg(rowptr + wr0) - kcta0, k1 = __ldg(rowptr + wr1) - kcta0;
    for (int r = wr0 + lane; r < wr1; r += 32) {
        double* yy = s_y + 3 * (r - rb);
        yy[0] = 0.0; yy[1] = 0.0; yy[2] = 0.0;
    }
    __syncwarp();
    for (int kb = k0; kb < k1; kb += 32 * NB) {
        CT p0[NB], p1[NB], p2[NB];
        int row[NB];
#pragma unroll
        for (int h = 0; h < NB; ++h) {
            const int k = kb + 32 * h + lane;
            row[h] = -1;
            p0[h] = 0; p1[h] = 0; p2[h] = 0;
            if (k < k1) {
                row[h] = s_lr[k];
                VT u0, u1, u2;
                Vec4<VT>::load(s_win, s_lc[k], u0, u1, u2);
                const CT x0 = (CT)u0, x1 = (CT)u1, x2 = (CT)u2;
                const MT* v = s_val + k;
                const CT b0 = Num<MT>::get(v[0]), b1 = Num<MT>::get(v[nblk]), b2 = Num<MT>::get(v[2 * nblk]),
                         b3 = Num<MT>::get(v[3 * nblk]), b4 = Num<MT>::get(v[4 * nblk]),
                         b5 = Num<MT>::get(v[5 * nblk]), b6 = Num<MT>::get(v[6 * nblk]),
                         b7 = Num<MT>::get(v[7 * nblk]), b8 = Num<MT>::get(v[8 * nblk]);
                p0[h] = dot3(b0, b1, b2, x0, x1, x2);
                p1[h] = dot3(b3, b4, b5, x0, x1, x2);
                p2[h] = dot3(b6, b7, b8, x0, x1, x2);
            }
        }
#pragma unroll
        for (int h = 0; h < NB; ++h) {
            CT a0 = p0[h], a1 = p1[h], a2 = p2[h];
            const int rw = row[h];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int rr = __shfl_up_sync(0xffffffffu, rw, off);
                const CT q0 = __shfl_up_sync(0xffffffffu, a0, off);
                const CT q1 = __shfl_up_sync(0xffffffffu, a1, off);
                const CT q2 = __shfl_up_sync(0xffffffffu, a2, off);
                if (lane >= off && rr == rw) { a0 += q0; a1 += q1; a2 += q2; }
            }
            const int rn = __shfl_down_sync(0xffffffffu, rw, 1);
            if (rw >= 0 && (lane == 31 || rn != rw)) {
                double* yy = s_y + 3 * rw;
                yy[0] += (double)a0; yy[1] += (double)a1; yy[2] += (double)a2;
            }
            __syncwarp();
        }
    }
    __syncwarp();
    for (int r = wr0 + lane; r < wr1; r += 32) {
        const double* yy = s_y + 3 * (r - rb);
        epi(r, (CT)yy[0], (CT)yy[1], (CT)yy[2]);
    }
}

// y_row = sum_k B_k x[col_k] from the CTA's shared-memory copy, four threads
// per row: each sums its blocks k = first + sub, + 4, ... in order, then a
// fixed butterfly adds the four partial sums; the sub == 0 thread runs the
// epilogue.  No scan: in shared memory the load pattern needs no warp-wide
// coalescing, and a row has ~12 blocks.
template <bool kGlobalVals, class MT, class CT, class VT, class Epi>
__device__ __forceinline__ void spmv_rows_res(int rb, int nrow, const int* s_rp, size_t pstride, const MT* val,
                                              const unsigned short* s_lc, const VT* s_win, Epi& epi) {
    // value planes: shared memory (val = the CTA's copy, pstride = its block
    // count) or global memory (val = the CTA's first block, pstride = nnz)
    auto ld = [&](const MT* p) -> CT { return (CT)Num<MT>::get(kGlobalVals ? __ldg(p) : *p); };
    const int sub = threadIdx.x & 3;
    for (int lr0 = 0; lr0 < nrow; lr0 += kThreads / 4) {
        const int lr = lr0 + (threadIdx.x >> 2);
        CT a0 = 0, a1 = 0, a2 = 0;
        if (lr < nrow) {
            const int k1 = s_rp[lr + 1];
            for (int k = s_rp[lr] + sub; k < k1; k += 4) {
                VT u0, u1, u2;
                Vec4<VT>::load(s_win, s_lc[k], u0, u1, u2);
                const CT x0 = (CT)u0, x1 = (CT)u1, x2 = (CT)u2;
                const MT* v = val + k;
                a0 += dot3(ld(v), ld(v + pstride), ld(v + 2 * pstride), x0, x1, x2);
                a1 += dot3(ld(v + 3 * pstride), ld(v + 4 * pstride), ld(v + 5 * pstride), x0, x1, x2);
                a2 += dot3(ld(v + 6 * pstride), ld(v + 7 * pstride), ld(v + 8 * pstride), x0, x1, x2);
            }
        }
        a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 1);
        a0 += __shfl_xor_sync(0xffffffffu, a0, 2);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 2);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 2);
        if (lr < nrow && sub == 0) epi(rb + lr, a0, a1, a2);
    }
}

template <class DT>
__device__ __forceinline__ void dinv_apply(const DT* __restrict__ dinv, int n, int row, double s,
                                           double r0, double r1, double r2, double& o0, double& o1, double& o2) {
    const DT* d = dinv + row;
    const double d0 = __ldg(d), d1 = __ldg(d + n), d2 = __ldg(d + 2 * (size_t)n);
    const double d3 = __ldg(d + 3 * (size_t)n), d4 = __ldg(d + 4 * (size_t)n), d5 = __ldg(d + 5 * (size_t)n);
    const double d6 = __ldg(d + 6 * (size_t)n), d7 = __ldg(d + 7 * (size_t)n), d8 = __ldg(d + 8 * (size_t)n);
    o0 = s * (d0 * r0 + d1 * r1 + d2 * r2);
    o1 = s * (d3 * r0 + d4 * r1 + d5 * r2);
    o2 = s * (d6 * r0 + d7 * r1 + d8 * r2);
}

// dinv_apply on the CTA's shared-memory copy of its rows' planes (stride = its row count)
template <class DT>
__device__ __forceinline__ void dinv_apply_s(const DT* sd, int stride, int lr, double s, double r0, double r1,
                                             double r2, double& o0, double& o1, double& o2) {
    const DT* d = sd + lr;
    const double d0 = d[0], d1 = d[stride], d2 = d[2 * stride], d3 = d[3 * stride], d4 = d[4 * stride];
    const double d5 = d[5 * stride], d6 = d[6 * stride], d7 = d[7 * stride], d8 = d[8 * stride];
    o0 = s * (d0 * r0 + d1 * r1 + d2 * r2);
    o1 = s * (d3 * r0 + d4 * r1 + d5 * r2);
    o2 = s * (d6 * r0 + d7 * r1 + d8 * r2);
}

enum SlotKind { kIdle = 0, kNormal = 1, kReplace = 2 };

template <class MT, class PT, class VT, int TPR>
__global__ void __launch_bounds__(kThreads, 1) pcg_kernel(const PcgParams prm_arg) {
    // The parameters and this CTA's system descriptor live in shared memory, one
    // copy per CTA: the lambdas below capture them by reference (a reference to
    // a kernel parameter would be a parameter-space address), and a per-thread
    // local copy (440 B x 512 threads) does not stay in L1, so its loads went to
    // L2 after every grid barrier.
    __shared__ __align__(16) unsigned char s_prm_raw[sizeof(PcgParams)];
    __shared__ __align__(16) unsigned char s_sys_raw[sizeof(SysDesc)];
    PcgParams& prm_sh = *reinterpret_cast<PcgParams*>(s_prm_raw);
    if (threadIdx.x == 0) prm_sh = prm_arg;
    __syncthreads();
    const PcgParams& prm = prm_sh;
    using CT = typename Cmp<MT>::T;
    using DT = typename DinvT<MT>::T;
    // 32-block slices a warp loads per round trip in the SpMV (the "tile width" the
    // autotuner picks through threads_per_row: 2 -> 1, 4 -> 2, 8 -> 4)
    constexpr int kNB = TPR / 2;
    // mixed modes keep the diagonal blocks of the coupled (active) nodes out of
    // the bulk planes and apply them in FP64: those blocks carry the contact /
    // stitch stiffness that cancels against the low-rank term in S = D - V C V^T
    constexpr bool kSplit = !std::is_same<MT, double>::value;
    __shared__ double s_w[kWarps][2];
    __shared__ double s_bc[4];
    __shared__ int s_ok;
    // this CTA's share of the tt_j = (Vt^T p)_j recurrence: columns j = lcta + ncta * q, their
    // partial-sum reads issued at the loop top by the warps idle there, their tt and d kept here
    __shared__ double s_zsum[kMaxRank], s_ttown[kMaxRank], s_dpown[kMaxRank];
    extern __shared__ __align__(16) double smem[];

    const int cta = blockIdx.x;
    const unsigned int G = gridDim.x;
    const int sidx = prm.cta_sys[cta];
    SysDesc& sys_sh = *reinterpret_cast<SysDesc*>(s_sys_raw);
    if (threadIdx.x == 0) sys_sh = prm.sys[sidx];
    __syncthreads();
    const SysDesc& S = sys_sh;
    const int rb = prm.cta_row[2 * cta], re = prm.cta_row[2 * cta + 1];
    const int ab = prm.cta_act[2 * cta], ae = prm.cta_act[2 * cta + 1];
    const int aidx = prm.cta_aidx[cta];
    const int na = ae - ab;
    const int cb = S.cta_begin, ce = S.cta_end;
    const int ncta = ce - cb, lcta = cta - cb;
    const bool leader_cta = (cta == cb);
    const int n = S.n, nnz = S.nnz, a = S.a;
    const int rank = *S.rank;
    const int tt_own = rank > lcta ? (rank - lcta + ncta - 1) / ncta : 0;  // columns this CTA reduces
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gwarp = lcta * kWarps + warp, nwarp = ncta * kWarps;
    const double omega = prm.omega;
    const int nterms = prm.nterms;
    const MT* vals = reinterpret_cast<const MT*>(S.vals);
    const PT* vals_pc = reinterpret_cast<const PT*>(S.vals_pc);
    const DT* dinv = reinterpret_cast<const DT*>(S.dinv);
    const double* vt = S.vt64;
    double* x = S.x;
    double* r = S.r;
    const double* rhs = S.rhs;
    VT* z = reinterpret_cast<VT*>(S.z);
    VT* y = reinterpret_cast<VT*>(S.y);
    // ping-pong buffers chosen by a select, not a runtime-indexed (local-memory) array
    VT* const pbuf0 = reinterpret_cast<VT*>(S.p[0]);
    VT* const pbuf1 = reinterpret_cast<VT*>(S.p[1]);
    VT* const tbuf0 = reinterpret_cast<VT*>(S.t[0]);
    VT* const tbuf1 = reinterpret_cast<VT*>(S.t[1]);
    auto pbuf = [&](int i) { return i ? pbuf1 : pbuf0; };
    auto tbuf = [&](int i) { return i ? tbuf1 : tbuf0; };

    // shared memory (offsets in doubles, the same in every CTA): d .* tt,
    // own coupled-dof z, the Vt block of the own coupled dofs, the row sums of
    // the SpMV, and the CTA's column indices and row ids
    double* s_dtt = smem;
    double* s_z = smem + prm.off_z;
    double* s_vt = smem + prm.off_vt;
    double* s_y = smem + prm.off_y;
    const int kcta0 = __ldg(S.rowptr + rb), nblk = __ldg(S.rowptr + re) - kcta0;
    int* s_col = prm.stage_blk ? reinterpret_cast<int*>(smem + prm.off_blk) : nullptr;
    int* s_row = prm.stage_blk ? s_col + nblk : nullptr;
    const int wr0 = prm.cta_warp[(kWarps + 1) * cta + warp], wr1 = prm.cta_warp[(kWarps + 1) * cta + warp + 1];
    if (s_col)
        for (int e = threadIdx.x; e < nblk; e += kThreads) {
            s_col[e] = __ldg(S.colidx + kcta0 + e);
            s_row[e] = __ldg(S.rowid + kcta0 + e);
        }
    // resident mode: the CTA's value planes, local indices and window node list
    const bool res = prm.resident != 0;
    const int wn0 = res ? prm.win_off[cta] : 0, nwin = res ? prm.win_off[cta + 1] - wn0 : 0;
    const int wown = res ? prm.win_own[cta] : 0;
    int* s_wn = reinterpret_cast<int*>(smem + prm.off_wn);
    VT* s_win = reinterpret_cast<VT*>(smem + prm.off_win);
    MT* s_val = reinterpret_cast<MT*>(smem + prm.off_val);
    PT* s_vpc = std::is_same<MT, PT>::value ? reinterpret_cast<PT*>(s_val) : reinterpret_cast<PT*>(smem + prm.off_vpc);
    unsigned short* s_lc = reinterpret_cast<unsigned short*>(smem + prm.off_lidx);
    unsigned short* s_lr = s_lc + nblk;
    const int nrow = re - rb;
    const int Rown = prm.own_rows, Zown = prm.own_act;
    DT* s_dinv = reinterpret_cast<DT*>(smem + prm.off_dinv);
    int* s_rf = reinterpret_cast<int*>(smem + prm.off_rf);
    int* s_rp = s_rf + Rown;   // the CTA's row pointers, local to its first block (nrow + 1)
    if (res) {
        if (prm.stage_vals)
            for (int e = threadIdx.x; e < 9 * nblk; e += kThreads) {
                const int pl = e / nblk, kl = e - pl * nblk;
                s_val[e] = vals[(size_t)pl * nnz + kcta0 + kl];
                if (!std::is_same<MT, PT>::value) s_vpc[e] = vals_pc[(size_t)pl * nnz + kcta0 + kl];
            }
        for (int e = threadIdx.x; e < nblk; e += kThreads) {
            s_lc[e] = S.lcol[kcta0 + e];
            s_lr[e] = (unsigned short)(__ldg(S.rowid + kcta0 + e) - rb);
        }
        for (int e = threadIdx.x; e < nwin; e += kThreads) s_wn[e] = prm.win_nodes[wn0 + e];
        for (int e = threadIdx.x; e < 9 * nrow; e += kThreads) {
            const int pl = e / nrow, lr = e - pl * nrow;
            s_dinv[e] = dinv[(size_t)pl * n + rb + lr];
        }
        for (int e = threadIdx.x; e < nrow; e += kThreads) s_rf[e] = __ldg(S.rowflag + rb + e);
        for (int e = threadIdx.x; e <= nrow; e += kThreads) s_rp[e] = __ldg(S.rowptr + rb + e) - kcta0;
    }
    // own-row vectors (resident mode): x, r, z, the new direction p, y = S p and
    // the current term t of the CTA's rows live in shared memory, 3 entries per
    // row; x, z, p and t are also written through to global memory, where the
    // neighbours' windows read them.  r and y never leave the CTA.
    double* s_xo = reinterpret_cast<double*>(smem + prm.off_own);
    double* s_ro = s_xo + 3 * Rown;
    VT* s_zo = reinterpret_cast<VT*>(s_ro + 3 * Rown);
    VT* s_po = s_zo + 3 * Rown;
    VT* s_yo = s_po + 3 * Rown;
    VT* s_to = s_yo + 3 * Rown;
    double* s_pa = reinterpret_cast<double*>(smem + prm.off_act);
    double* s_ya = s_pa + Zown;
    int* s_act = reinterpret_cast<int*>(s_ya + Zown);
    if (res)
        for (int e = threadIdx.x; e < na; e += kThreads) s_act[e] = __ldg(S.act + ab + e);
    // fused update: window flags, the coupled window nodes and their corrections
    const bool fuse = res && prm.fuse != 0;
    int* s_wflag = reinterpret_cast<int*>(smem + prm.off_wflag);
    int* s_wan = reinterpret_cast<int*>(smem + prm.off_wact);
    double* s_wcorr = smem + prm.off_wcorr;
    const int wa0 = fuse ? prm.win_act_off[cta] : 0, nwa = fuse ? prm.win_act_off[cta + 1] - wa0 : 0;
    if (fuse) {
        for (int e = threadIdx.x; e < nwin; e += kThreads) s_wflag[e] = prm.win_flag[wn0 + e];
        for (int e = threadIdx.x; e < nwa; e += kThreads) s_wan[e] = prm.win_act[wa0 + e];
    }
    double* rbuf[2] = {S.r, S.r2};
    int rcur = 0;      // residual buffer the neighbours read (fused update)
    int tail_k0 = 1;   // first preconditioner phase the next precond_tail runs
    auto ld_z = [&](int row, VT& a0, VT& a1, VT& a2) {
        if (res) { const VT* q = s_zo + 3 * (row - rb); a0 = q[0]; a1 = q[1]; a2 = q[2]; }
        else Vec4<VT>::load(z, row, a0, a1, a2);
    };
    auto st_z = [&](int row, VT a0, VT a1, VT a2) {
        Vec4<VT>::store(z, row, a0, a1, a2);
        if (res) { VT* q = s_zo + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2; }
    };
    auto ld_r = [&](int row, double& a0, double& a1, double& a2) {
        if (res) { const double* q = s_ro + 3 * (row - rb); a0 = q[0]; a1 = q[1]; a2 = q[2]; }
        else Vec4<double>::load(r, row, a0, a1, a2);
    };
    auto st_r = [&](int row, double a0, double a1, double a2) {
        if (res) {
            double* q = s_ro + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2;
            if (fuse) Vec4<double>::store(rbuf[rcur], row, a0, a1, a2);
        } else {
            Vec4<double>::store(r, row, a0, a1, a2);
        }
    };
    auto ld_x = [&](int row, double& a0, double& a1, double& a2) {
        if (res) { const double* q = s_xo + 3 * (row - rb); a0 = q[0]; a1 = q[1]; a2 = q[2]; }
        else Vec4<double>::load(x, row, a0, a1, a2);
    };
    auto st_x = [&](int row, double a0, double a1, double a2) {
        Vec4<double>::store(x, row, a0, a1, a2);
        if (res) { double* q = s_xo + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2; }
    };
    auto ld_p = [&](const VT* pg, int row, VT& a0, VT& a1, VT& a2) {
        if (res) { const VT* q = s_po + 3 * (row - rb); a0 = q[0]; a1 = q[1]; a2 = q[2]; }
        else Vec4<VT>::load(pg, row, a0, a1, a2);
    };
    auto st_p = [&](VT* pg, int row, VT a0, VT a1, VT a2) {
        Vec4<VT>::store(pg, row, a0, a1, a2);
        if (res) { VT* q = s_po + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2; }
    };
    auto ld_y = [&](int row, VT& a0, VT& a1, VT& a2) {
        if (res) { const VT* q = s_yo + 3 * (row - rb); a0 = q[0]; a1 = q[1]; a2 = q[2]; }
        else Vec4<VT>::load(y, row, a0, a1, a2);
    };
    auto st_y = [&](int row, VT a0, VT a1, VT a2) {
        if (res) { VT* q = s_yo + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2; }
        if (!res || fuse) Vec4<VT>::store(y, row, a0, a1, a2);
    };
    auto st_t = [&](VT* tg, int row, VT a0, VT a1, VT a2) {
        Vec4<VT>::store(tg, row, a0, a1, a2);
        if (res) { VT* q = s_to + 3 * (row - rb); q[0] = a0; q[1] = a1; q[2] = a2; }
    };
    // direction / product at the coupled dofs (index i in the system's act list)
    auto pact_ref = [&](int i) -> double& { return res ? s_pa[i - ab] : S.pact[i]; };
    auto yact_ref = [&](int i) -> double& { return res ? s_ya[i - ab] : S.yact[i]; };
    // rowflag / Dd^-1 of an own row: shared-memory copies in resident mode
    auto rowflag_of = [&](int row) -> int { return res ? s_rf[row - rb] : __ldg(S.rowflag + row); };
    auto dinv_row = [&](int row, double r0, double r1, double r2, double& o0, double& o1, double& o2) {
        if (res) dinv_apply_s(s_dinv, nrow, row - rb, omega, r0, r1, r2, o0, o1, o2);
        else dinv_apply(dinv, n, row, omega, r0, r1, r2, o0, o1, o2);
    };
    // stage node values into the window: every thread issues the loads of up
    // to four (FP64: two) nodes before it stores any, so the window costs one
    // round trip
    auto stage_window = [&](auto&& load_node) {
        constexpr int SQ = sizeof(VT) == 8 ? 2 : 4;
        for (int i0 = threadIdx.x; i0 < nwin; i0 += SQ * kThreads) {
            VT v[SQ][3];
#pragma unroll
            for (int q = 0; q < SQ; ++q) {
                const int i = i0 + q * kThreads;
                if (i < nwin) load_node(s_wn[i], v[q][0], v[q][1], v[q][2]);
            }
#pragma unroll
            for (int q = 0; q < SQ; ++q) {
                const int i = i0 + q * kThreads;
                if (i < nwin) Vec4<VT>::store(s_win, i, v[q][0], v[q][1], v[q][2]);
            }
        }
    };
    const bool vt_smem = prm.stage_vt && na > 0;
    HSC_IN(rank <= kMaxRank && rank <= S.kmax, 207, rank);
    HSC_IN(na <= 0 || ((na + 1) & ~1) + na * rank <= prm.vt_smem, 201, na);
    if (vt_smem)
        for (int e = threadIdx.x; e < na * rank; e += kThreads) {
            const int j = e / na, il = e - j * na;
            if (HSC_IN(e < prm.vt_smem && ab + il < a, 200, e))
                s_vt[e] = __ldg(vt + (size_t)j * a + ab + il);
        }
    __syncthreads();
    auto vt_own = [&](int j, int il) -> double {
        return vt_smem ? s_vt[j * na + il] : __ldg(vt + (size_t)j * a + ab + il);
    };

    int it = 0, status = 0, nrep = 0;
    double rz = 0.0, normb = 0.0, rel = 1.0, beta = 0.0;
    bool done = false, counted = false, first = true;
    int slot = kNormal, prev_slot = kNormal;
    bool conv_check = false;
    int pc = 0;  // p buffer holding the previous direction
    int tc = 0;  // t buffer holding the current term
    int epoch = 0;
    int slot_no = 0;  // main-loop slots executed (trace index)
    auto mark = [&](int ev) {
        if (prm.trace && threadIdx.x == 0 && slot_no < prm.trace_iters)
            prm.trace[((size_t)cta * prm.trace_iters + slot_no) * kTraceEvents + ev] = (unsigned long long)clock64();
    };

    // grid barrier with the CTA partials folded into the arrival: each warp
    // reduces its values, thread 0 adds the warp sums (fixed order), stores
    // them and arrives
    auto barrier = [&](double* o0, double v0, double* o1, double v1) -> bool {
        v0 = warp_sum(v0);
        v1 = warp_sum(v1);
        if (lane == 0) { s_w[warp][0] = v0; s_w[warp][1] = v1; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double t0 = 0.0, t1 = 0.0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) { t0 += s_w[w][0]; t1 += s_w[w][1]; }
            if (o0) o0[cta] = t0;
            if (o1) o1[cta] = t1;
            s_ok = grid_arrive_wait(prm.bar, G, prm.spin_limit, epoch);
        }
        ++epoch;
        __syncthreads();
        return s_ok != 0;
    };
    auto dact_mul = [&](int an, double p0, double p1, double p2, double& o0, double& o1, double& o2) {
        const double* d = S.dact + 9 * (size_t)an;
        o0 = d[0] * p0 + d[1] * p1 + d[2] * p2;
        o1 = d[3] * p0 + d[4] * p1 + d[5] * p2;
        o2 = d[6] * p0 + d[7] * p1 + d[8] * p2;
    };
    // per-CTA partials of Vt^T v over the CTA's own coupled dofs (v final),
    // written to dst[j * stride]
    auto compute_part = [&](void* v, const VT* vown, double* dst, int stride) {
        if (na <= 0) return;  // uniform within the CTA
        __syncthreads();
        for (int il = threadIdx.x; il < na; il += kThreads) {
            if (res) {
                s_z[il] = (double)vown[s_act[il] - 3 * rb];
            } else {
                const int dof = __ldg(S.act + ab + il);
                if (HSC_IN(dof >= 0 && dof < 3 * n, 204, dof)) s_z[il] = (double)elem<VT>(v, dof);
            }
        }
        __syncthreads();
        // JW columns per warp, the first 128 coupled dofs fully unrolled so every
        // Vt load of the warp is in flight at once (one round trip when Vt is
        // read from L2); the summation order per column is il = lane, +32, ...
        constexpr int JW = 6;
        for (int j0 = warp * JW; j0 < rank; j0 += kWarps * JW) {
            double sacc[JW];
#pragma unroll
            for (int q = 0; q < JW; ++q) sacc[q] = 0.0;
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int il = lane + 32 * m;
                if (il < na) {
                    const double zv = s_z[il];
#pragma unroll
                    for (int q = 0; q < JW; ++q)
                        if (j0 + q < rank) sacc[q] += vt_own(j0 + q, il) * zv;
                }
            }
            for (int il = lane + 128; il < na; il += 32) {
                const double zv = s_z[il];
#pragma unroll
                for (int q = 0; q < JW; ++q)
                    if (j0 + q < rank) sacc[q] += vt_own(j0 + q, il) * zv;
            }
#pragma unroll
            for (int q = 0; q < JW; ++q) {
                const double t = warp_sum(sacc[q]);
                if (lane == 0 && j0 + q < rank && HSC_IN(j0 + q < S.kmax, 205, j0 + q)) dst[(size_t)(j0 + q) * stride] = t;
            }
        }
    };
    auto compute_zpart = [&]() { compute_part(z, s_zo, S.zpart + lcta, ncta); };
    const bool schur = prm.schur_basis != 0;
    const int nact = S.nact_cta;
    auto tpart_half = [&](int h) { return S.tpart + (size_t)h * S.kmax * nact; };
    // s_dtt[j] = d_j * sum_c P[j * nact + c] for j < rank: the partials of the
    // coupled CTAs, JW rows per warp with all their loads issued together,
    // summed in the same order in every CTA
    auto sum_tparts = [&](const double* P) {
        constexpr int JW = 8;
        // the warps take the column groups in an order rotated by the CTA, so the coupled CTAs do not
        // all read the same partials at the same moment
        const int ngroups = (rank + JW - 1) / JW;
        for (int g = warp; g < ngroups; g += kWarps) {
            const int j0 = ((g + aidx) % ngroups) * JW;
            double v[JW];
#pragma unroll
            for (int q = 0; q < JW; ++q) v[q] = 0.0;
            for (int c = lane; c < nact; c += 32)
#pragma unroll
                for (int q = 0; q < JW; ++q)
                    if (j0 + q < rank) v[q] += P[(size_t)(j0 + q) * nact + c];
#pragma unroll
            for (int q = 0; q < JW; ++q) {
                const double t = warp_sum(v[q]);
                if (lane == 0 && j0 + q < rank) s_dtt[j0 + q] = __ldg(S.dpiv + j0 + q) * t;
            }
        }
    };
    // out[il] = sum_j Vt[own il, j] s_dtt[j] for il < na: eight threads per
    // row (j interleaved; the first 128 columns fully unrolled so all loads are
    // in flight at once), combined by shuffles in a fixed order
    auto lowrank_rows = [&](double* out) {
        for (int base = 0; base < na; base += kThreads / 8) {
            const int il = base + (threadIdx.x >> 3), q = threadIdx.x & 7;
            double c = 0.0;
            if (il < na) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int j = q + 8 * m;
                    if (j < rank) c += vt_own(j, il) * s_dtt[j];
                }
                for (int j = q + 128; j < rank; j += 8) c += vt_own(j, il) * s_dtt[j];
            }
            c += __shfl_xor_sync(0xffffffffu, c, 1);
            c += __shfl_xor_sync(0xffffffffu, c, 2);
            c += __shfl_xor_sync(0xffffffffu, c, 4);
            if (il < na && q == 0) out[il] = c;
        }
    };
    const double* wdev = S.wdev;
    auto weight = [&](int k) -> double { return wdev ? wdev[k] : prm.w[k]; };
    // C_k phases k = 1..nterms-1 of the preconditioner polynomial
    auto precond_tail = [&](bool active_sys) -> bool {
        for (int k = tail_k0; k < nterms; ++k) {
            double acc = 0.0;
            const bool last = (k == nterms - 1);
            if (active_sys) {
                const VT* tcur = tbuf(tc);
                VT* tnew = tbuf(tc ^ 1);
                const double wk = weight(k);
                // Schur basis: low-rank part Vt d Vt^T t of S t at the own coupled dofs
                const bool corr = schur && na > 0;
                if (corr) {
                    sum_tparts(tpart_half((k - 1) & 1));
                    __syncthreads();
                    lowrank_rows(s_z);
                    __syncthreads();
                }
                auto gather = [&](int c, CT& g0, CT& g1, CT& g2) {
                    VT u0, u1, u2;
                    Vec4<VT>::load(tcur, c, u0, u1, u2);
                    g0 = (CT)u0; g1 = (CT)u1; g2 = (CT)u2;
                };
                auto epi = [&](int row, CT w0, CT w1, CT w2) {
                    VT c0, c1, c2;
                    if (res) Vec4<VT>::load(s_win, wown + row - rb, c0, c1, c2);
                    else Vec4<VT>::load(tcur, row, c0, c1, c2);
                    double v0 = w0, v1 = w1, v2 = w2;
                    if (kSplit) {
                        const int an = rowflag_of(row);
                        if (an >= 0) {
                            double d0, d1, d2;
                            dact_mul(an, (double)c0, (double)c1, (double)c2, d0, d1, d2);
                            v0 += d0; v1 += d1; v2 += d2;
                        }
                    }
                    if (corr) {
                        const int an = rowflag_of(row);
                        if (an >= 0) {
                            const int il = 3 * an - ab;
                            if (HSC_IN(il >= 0 && il + 2 < na, 208, il)) {
                                v0 -= s_z[il]; v1 -= s_z[il + 1]; v2 -= s_z[il + 2];
                            }
                        }
                    }
                    double e0, e1, e2;
                    dinv_row(row, v0, v1, v2, e0, e1, e2);
                    const double n0 = (double)c0 - e0, n1 = (double)c1 - e1, n2 = (double)c2 - e2;
                    st_t(tnew, row, (VT)n0, (VT)n1, (VT)n2);
                    VT q0, q1, q2;
                    ld_z(row, q0, q1, q2);
                    const VT s0 = (VT)((double)q0 + wk * n0), s1 = (VT)((double)q1 + wk * n1),
                             s2 = (VT)((double)q2 + wk * n2);
                    st_z(row, s0, s1, s2);
                    if (last) {
                        double r0, r1, r2;
                        ld_r(row, r0, r1, r2);
                        acc += r0 * (double)s0 + r1 * (double)s1 + r2 * (double)s2;
                    }
                };
                if (res) {
                    stage_window([&](int node, VT& u0, VT& u1, VT& u2) { Vec4<VT>::load(tcur, node, u0, u1, u2); });
                    __syncthreads();
                    if (last) mark(7);
                    if (prm.stage_vals) spmv_rows_res<false, PT, CT, VT>(rb, nrow, s_rp, nblk, s_vpc, s_lc, s_win, epi);
                    else spmv_rows_res<true, PT, CT, VT>(rb, nrow, s_rp, (size_t)nnz, vals_pc + kcta0, s_lc, s_win, epi);
                } else {
                    if (last) mark(7);
                    spmv_warp<kNB, PT, CT>(wr0, wr1, rb, S.rowptr, S.colidx, S.rowid, s_col, s_row, kcta0, vals_pc, nnz, s_y,
                                      gather, epi);
                }
                __syncthreads();
                if (last) mark(8);
                if (last) compute_zpart();
                else if (schur) compute_part(tnew, s_to, tpart_half(k & 1) + aidx, nact);
            }
            tc ^= 1;
            if (last) mark(5);
            if (!barrier(last ? prm.part_rz : nullptr, acc, nullptr, 0.0)) return false;
            if (last) mark(6);
        }
        return true;
    };

    // ---------------- prologue: r = rhs, x = 0, z = M r ----------------
    {
        for (int q = threadIdx.x; q < tt_own; q += kThreads) {
            s_ttown[q] = 0.0;
            s_dpown[q] = __ldg(S.dpiv + lcta + (size_t)ncta * q);
        }
        double acc_rr = 0.0, acc_rz = 0.0;
        for (int row = rb + threadIdx.x; row < re; row += kThreads) {
            double r0, r1, r2;
            Vec4<double>::load(rhs, row, r0, r1, r2);
            st_r(row, r0, r1, r2);
            st_x(row, 0.0, 0.0, 0.0);
            Vec4<VT>::store(pbuf(0), row, (VT)0, (VT)0, (VT)0);  // beta * p_prev must be 0, not NaN
            double t0, t1, t2;
            dinv_row(row, r0, r1, r2, t0, t1, t2);
            st_t(tbuf(0), row, (VT)t0, (VT)t1, (VT)t2);
            const double w0 = weight(0);
            const VT z0 = (VT)(w0 * t0), z1 = (VT)(w0 * t1), z2 = (VT)(w0 * t2);
            st_z(row, z0, z1, z2);
            acc_rr += r0 * r0 + r1 * r1 + r2 * r2;
            acc_rz += r0 * (double)z0 + r1 * (double)z1 + r2 * (double)z2;
        }
        for (int i = ab + threadIdx.x; i < ae; i += kThreads) pact_ref(i) = 0.0;
        if (na <= 0)
            for (int j = threadIdx.x; j < rank; j += kThreads) S.zpart[(size_t)j * ncta + lcta] = 0.0;
        if (schur && nterms > 1) compute_part(tbuf(0), s_to, tpart_half(0) + aidx, nact);
        if (leader_cta)
            for (int j = threadIdx.x; j < rank; j += kThreads) S.tt[j] = 0.0;
        if (nterms == 1) compute_zpart();
        if (!barrier(prm.part_rr, acc_rr, nterms == 1 ? prm.part_rz : nullptr, acc_rz)) return;
    }
    // ---------------- main loop: one slot per iteration ----------------
    // The preconditioner phases of a slot run at the top of the next loop pass
    // (the first pass: those of the prologue), so precond_tail has one call
    // site: the kernel stays small enough for the compiler to keep it inline.
    bool tail_active = true;
    for (;;) {
        if (!precond_tail(tail_active)) return;
        mark(0);
        if (warp == 0) {
            double srr, srz;
            warp_sum_parts(prm.part_rr, prm.part_rz, cb, ce, srr, srz);
            if (lane == 0) { s_bc[0] = srr; s_bc[1] = srz; }
        } else {
            // the other warps read this CTA's columns of the per-CTA Vt^T z partials (final since the
            // preconditioner's barrier) in the same round trip; used by phase A of a normal slot
            for (int q = warp - 1; q < tt_own; q += kWarps - 1) {
                double sz, unused;
                warp_sum_parts(S.zpart + (size_t)(lcta + ncta * q) * ncta, nullptr, 0, ncta, sz, unused);
                if (lane == 0) s_zsum[q] = sz;
            }
        }
        mark(14);
        __syncthreads();
        const double rr = s_bc[0];
        const double rzn = s_bc[1];
        if (!done) {
            if (first) {
                normb = sqrt(rr);
                rel = normb > 0 ? 1.0 : 0.0;
                if (!(normb > 0)) { done = true; status = 0; }
                if (!isfinite(normb)) { done = true; status = 3; }
            } else {
                rel = sqrt(rr) / normb;
            }
            if (!done) {
                if (prev_slot == kReplace) {
                    ++nrep;
                    if (rel <= prm.tol) { done = true; status = 0; }
                    else if (it >= prm.max_iter) { done = true; status = 4; }
                    else {
                        beta = conv_check ? 0.0 : rzn / rz;                    // restart after a failed check
                        slot = kNormal;
                    }
                    conv_check = false;
                } else if (!first && rel <= prm.tol) {
                    slot = kReplace; conv_check = true;                        // linear_hsc.cu:375-387
                } else if (it >= prm.max_iter) {
                    done = true; status = 4;
                } else if (!first && prm.rr_every > 0 && it % prm.rr_every == 0) {
                    slot = kReplace; conv_check = false;                       // FP64 reliable update
                } else {
                    beta = first ? 0.0 : rzn / rz;
                    slot = kNormal;
                }
                if (!done && slot == kNormal) {
                    if (!(isfinite(rzn) && rzn > 0)) { done = true; status = 3; }   // linear_hsc.cu:370-371
                    else rz = rzn;
                    if (!done && leader_cta && threadIdx.x == 0 && it < S.max_coef && it > 0)
                        S.cg_coef[2 * (it - 1) + 1] = beta;
                }
            }
            first = false;
        }
        if (done) slot = kIdle;
        if (done && !counted) {
            counted = true;
            if (leader_cta && threadIdx.x == 0) {
                S.out[0] = it; S.out[1] = rel; S.out[2] = status; S.out[3] = normb; S.out[4] = nrep;
                __threadfence();
                atomicSub(prm.remaining, 1);
            }
        }

        mark(15);
        // ---- phase A: y = D p (p = z + beta p_prev on the fly), tt = Vt^T p ----
        {
            double acc = 0.0;
            if (slot == kNormal) {
                VT* pnew = pbuf(pc ^ 1);
                const VT* pprev = pbuf(pc);
                const CT bc = (CT)beta;
                const double bd = beta;
                auto gather = [&](int c, CT& g0, CT& g1, CT& g2) {
                    VT z0, z1, z2, q0, q1, q2;
                    if (!HSC_IN(c >= 0 && c < n, 203, c)) c = 0;
                    Vec4<VT>::load(z, c, z0, z1, z2);
                    Vec4<VT>::load(pprev, c, q0, q1, q2);
                    g0 = (CT)(VT)((CT)z0 + bc * (CT)q0);
                    g1 = (CT)(VT)((CT)z1 + bc * (CT)q1);
                    g2 = (CT)(VT)((CT)z2 + bc * (CT)q2);
                };
                auto epi = [&](int row, CT y0, CT y1, CT y2) {
                    CT g0, g1, g2;
                    if (res) {
                        VT u0, u1, u2;
                        Vec4<VT>::load(s_win, wown + row - rb, u0, u1, u2);
                        g0 = (CT)u0; g1 = (CT)u1; g2 = (CT)u2;
                    } else {
                        gather(row, g0, g1, g2);
                    }
                    st_p(pnew, row, (VT)g0, (VT)g1, (VT)g2);
                    int an = rowflag_of(row);
                    if (!HSC_IN(an < a / 3, 206, an)) an = -1;
                    if (an >= 0) {
                        // FP64 direction and product at a coupled node
                        VT z0, z1, z2;
                        ld_z(row, z0, z1, z2);
                        double& pa0 = pact_ref(3 * an);
                        double& pa1 = pact_ref(3 * an + 1);
                        double& pa2 = pact_ref(3 * an + 2);
                        const double a0 = (double)z0 + bd * pa0, a1 = (double)z1 + bd * pa1, a2 = (double)z2 + bd * pa2;
                        pa0 = a0; pa1 = a1; pa2 = a2;
                        double v0 = y0, v1 = y1, v2 = y2;
                        if (kSplit) {
                            double d0, d1, d2;
                            dact_mul(an, a0, a1, a2, d0, d1, d2);
                            v0 += d0; v1 += d1; v2 += d2;
                        }
                        yact_ref(3 * an) = v0; yact_ref(3 * an + 1) = v1; yact_ref(3 * an + 2) = v2;
                        if (fuse) { double* yg = S.yact + 3 * (size_t)an; yg[0] = v0; yg[1] = v1; yg[2] = v2; }
                        acc += a0 * v0 + a1 * v1 + a2 * v2;
                    } else {
                        st_y(row, (VT)y0, (VT)y1, (VT)y2);
                        acc += (double)g0 * (double)(VT)y0 + (double)g1 * (double)(VT)y1 + (double)g2 * (double)(VT)y2;
                    }
                };
                if (res) {
                    // stage p = z + beta p_prev over the window, then the SpMV from shared memory
                    stage_window([&](int node, VT& u0, VT& u1, VT& u2) {
                        CT g0, g1, g2;
                        gather(node, g0, g1, g2);
                        u0 = (VT)g0; u1 = (VT)g1; u2 = (VT)g2;
                    });
                    __syncthreads();
                    mark(9);
                    if (prm.stage_vals) spmv_rows_res<false, MT, CT, VT>(rb, nrow, s_rp, nblk, s_val, s_lc, s_win, epi);
                    else spmv_rows_res<true, MT, CT, VT>(rb, nrow, s_rp, (size_t)nnz, vals + kcta0, s_lc, s_win, epi);
                } else {
                    mark(9);
                    spmv_warp<kNB, MT, CT>(wr0, wr1, rb, S.rowptr, S.colidx, S.rowid, s_col, s_row, kcta0, vals, nnz, s_y,
                                      gather, epi);
                }
                __syncthreads();
                mark(10);
                // tt_j = (Vt^T z)_j + beta tt_j for this CTA's columns (sums read at the loop top)
                for (int q = threadIdx.x; q < tt_own; q += kThreads) {
                    const double t = s_zsum[q] + bd * s_ttown[q];
                    s_ttown[q] = t;
                    S.tt[lcta + (size_t)ncta * q] = t;
                    acc -= s_dpown[q] * t * t;
                }
            } else if (slot == kReplace) {
                // r = rhs - D x in FP64 (the assembled matrix, not the bulk precision)
                auto gather = [&](int c, double& g0, double& g1, double& g2) { Vec4<double>::load(x, c, g0, g1, g2); };
                auto epi = [&](int row, double y0, double y1, double y2) {
                    double h0, h1, h2;
                    Vec4<double>::load(rhs, row, h0, h1, h2);
                    st_r(row, h0 - y0, h1 - y1, h2 - y2);
                };
                spmv_warp<kNB, double, double>(wr0, wr1, rb, S.rowptr, S.colidx, S.rowid, s_col, s_row, kcta0, S.vals64, nnz, s_y, gather, epi);
                for (int j = gwarp; j < rank; j += nwarp) {
                    const double* col = vt + (size_t)j * a;
                    double d = 0.0;
                    for (int i = lane; i < a; i += 32) {
                        const int dof = __ldg(S.act + i);
                        d += __ldg(col + i) * x[4 * (dof / 3) + dof % 3];
                    }
                    d = warp_sum(d);
                    if (lane == 0) S.ttx[j] = d;
                }
            }
            mark(1);
            if (!barrier(prm.part_pap, acc, nullptr, 0.0)) return;
            mark(2);
        }
        // every system finished: only possible once this CTA's own system is done, so the
        // load stays off the critical path of the CTAs still iterating
        if (done && ld_volatile_i32(prm.remaining) == 0) break;

        // ---- phase B: alpha, low-rank correction, x/r update, t = w Dd^-1 r ----
        {
            double acc_rr = 0.0, acc_rz = 0.0;
            bool work = slot != kIdle;
            double alpha = 0.0;
            // the coupled-dof CTAs read d .* tt (or d .* ttx) while warp 0 sums the partials
            const bool fused_slot = fuse && slot == kNormal;
            if (slot != kIdle && (na > 0 || (fused_slot && nwa > 0))) {
                const double* tsrc = slot == kNormal ? S.tt : S.ttx;
                for (int j = (int)threadIdx.x - 32; j < rank; j += kThreads - 32)
                    if (j >= 0) s_dtt[j] = __ldg(S.dpiv + j) * tsrc[j];
            }
            if (slot == kNormal) {
                if (warp == 0) {
                    double sp, unused;
                    warp_sum_parts(prm.part_pap, nullptr, cb, ce, sp, unused);
                    if (lane == 0) s_bc[2] = sp;
                }
                __syncthreads();
                mark(11);
                const double pAp = s_bc[2];
                if (!(isfinite(pAp) && pAp > 0)) {
                    done = true; status = 3; work = false;                      // linear_hsc.cu:370-371
                } else {
                    alpha = rz / pAp;
                    if (leader_cta && threadIdx.x == 0 && it < S.max_coef) S.cg_coef[2 * it] = alpha;
                }
            }
            if (work && fused_slot) {
                // ---- fused update + first preconditioner phase ----
                const VT* pnew = pbuf(pc ^ 1);
                const double W0 = weight(0), W1 = weight(1);
                const bool last1 = nterms == 2;
                const double* rold = rbuf[rcur];
                double* rnew = rbuf[rcur ^ 1];
                VT* t1buf = tbuf(tc ^ 1);
                __syncthreads();  // s_dtt filled above
                // low-rank part of y at the coupled window dofs: 8 threads per dof
                // (the order of lowrank_rows), Vt rows read from L2
                for (int base = 0; base < 3 * nwa; base += kThreads / 8) {
                    const int e = base + (threadIdx.x >> 3), q = threadIdx.x & 7;
                    double c = 0.0;
                    if (e < 3 * nwa) {
                        const double* vrow = vt + 3 * s_wan[e / 3] + e % 3;
#pragma unroll
                        for (int m = 0; m < 16; ++m) {
                            const int j = q + 8 * m;
                            if (j < rank) c += __ldg(vrow + (size_t)j * a) * s_dtt[j];
                        }
                        for (int j = q + 128; j < rank; j += 8) c += __ldg(vrow + (size_t)j * a) * s_dtt[j];
                    }
                    c += __shfl_xor_sync(0xffffffffu, c, 1);
                    c += __shfl_xor_sync(0xffffffffu, c, 2);
                    c += __shfl_xor_sync(0xffffffffu, c, 4);
                    if (e < 3 * nwa && q == 0) s_wcorr[e] = c;
                }
                __syncthreads();
                mark(12);
                // y_full at a window node (S p with the low-rank term)
                auto y_full = [&](int wi, int node, double& y0, double& y1, double& y2) {
                    const int k = s_wflag[wi];
                    if (k >= 0) {
                        const double* yg = S.yact + 3 * (size_t)s_wan[k];
                        y0 = yg[0] - s_wcorr[3 * k]; y1 = yg[1] - s_wcorr[3 * k + 1]; y2 = yg[2] - s_wcorr[3 * k + 2];
                    } else {
                        VT u0, u1, u2;
                        Vec4<VT>::load(y, node, u0, u1, u2);
                        y0 = u0; y1 = u1; y2 = u2;
                    }
                };
                // t0 = w Dd^-1 (r - alpha y) over the window, the same arithmetic in every CTA
                for (int wi = threadIdx.x; wi < nwin; wi += kThreads) {
                    const int node = s_wn[wi];
                    double y0, y1, y2, r0, r1, r2, t0, t1, t2;
                    y_full(wi, node, y0, y1, y2);
                    Vec4<double>::load(rold, node, r0, r1, r2);
                    r0 -= alpha * y0; r1 -= alpha * y1; r2 -= alpha * y2;
                    dinv_apply(dinv, n, node, omega, r0, r1, r2, t0, t1, t2);
                    Vec4<VT>::store(s_win, wi, (VT)t0, (VT)t1, (VT)t2);
                }
                __syncthreads();
                double acc_rr2 = 0.0, acc_rz2 = 0.0;
                auto epi = [&](int row, CT w0, CT w1, CT w2) {
                    const int lr = row - rb;
                    double y0, y1, y2, p0, p1, p2;
                    y_full(wown + lr, row, y0, y1, y2);
                    const int an = rowflag_of(row);
                    if (an >= 0) {
                        p0 = pact_ref(3 * an); p1 = pact_ref(3 * an + 1); p2 = pact_ref(3 * an + 2);
                    } else {
                        VT q0, q1, q2;
                        ld_p(pnew, row, q0, q1, q2);
                        p0 = q0; p1 = q1; p2 = q2;
                    }
                    double x0, x1, x2, r0, r1, r2;
                    ld_x(row, x0, x1, x2);
                    Vec4<double>::load(rold, row, r0, r1, r2);
                    x0 += alpha * p0; x1 += alpha * p1; x2 += alpha * p2;
                    r0 -= alpha * y0; r1 -= alpha * y1; r2 -= alpha * y2;
                    st_x(row, x0, x1, x2);
                    { double* q = s_ro + 3 * lr; q[0] = r0; q[1] = r1; q[2] = r2; }
                    Vec4<double>::store(rnew, row, r0, r1, r2);
                    double d0, d1, d2;
                    dinv_row(row, r0, r1, r2, d0, d1, d2);                 // t0 in FP64
                    const VT c0 = (VT)d0, c1 = (VT)d1, c2 = (VT)d2;        // == the window copy
                    const VT zb0 = (VT)(W0 * d0), zb1 = (VT)(W0 * d1), zb2 = (VT)(W0 * d2);
                    double v0 = w0, v1 = w1, v2 = w2;
                    if (kSplit && an >= 0) {
                        double e0, e1, e2;
                        dact_mul(an, (double)c0, (double)c1, (double)c2, e0, e1, e2);
                        v0 += e0; v1 += e1; v2 += e2;
                    }
                    double e0, e1, e2;
                    dinv_row(row, v0, v1, v2, e0, e1, e2);
                    const double n0 = (double)c0 - e0, n1 = (double)c1 - e1, n2 = (double)c2 - e2;
                    st_t(t1buf, row, (VT)n0, (VT)n1, (VT)n2);
                    const VT s0 = (VT)((double)zb0 + W1 * n0), s1 = (VT)((double)zb1 + W1 * n1),
                             s2 = (VT)((double)zb2 + W1 * n2);
                    st_z(row, s0, s1, s2);
                    acc_rr2 += r0 * r0 + r1 * r1 + r2 * r2;
                    if (last1) acc_rz2 += r0 * (double)s0 + r1 * (double)s1 + r2 * (double)s2;
                };
                if (prm.stage_vals) spmv_rows_res<false, PT, CT, VT>(rb, nrow, s_rp, nblk, s_vpc, s_lc, s_win, epi);
                else spmv_rows_res<true, PT, CT, VT>(rb, nrow, s_rp, (size_t)nnz, vals_pc + kcta0, s_lc, s_win, epi);
                __syncthreads();
                mark(13);
                if (last1) compute_zpart();
                acc_rr = acc_rr2;
                acc_rz = acc_rz2;
                ++it;
                pc ^= 1;
                rcur ^= 1;
                tc ^= 1;
            } else if (work) {
                if (na > 0) {
                    __syncthreads();  // s_dtt filled above
                    lowrank_rows(s_z);
                    __syncthreads();
                    mark(12);
                    for (int il = threadIdx.x; il < na; il += kThreads) {
                        const double c = s_z[il];
                        if (slot == kNormal) yact_ref(ab + il) -= c;                   // y = D p - Vt d Vt^T p
                        else if (res) {                                                // r = rhs - D x + Vt d Vt^T x
                            const int dl = s_act[il] - 3 * rb;
                            s_ro[dl] += c;
                            if (fuse) rbuf[rcur][4 * (s_act[il] / 3) + s_act[il] % 3] = s_ro[dl];
                        }
                        else elem<double>(r, __ldg(S.act + ab + il)) += c;
                    }
                }
                __syncthreads();
                const VT* pnew = pbuf(pc ^ 1);
                const double w0 = weight(0);
                for (int row = rb + threadIdx.x; row < re; row += kThreads) {
                    double r0, r1, r2;
                    if (slot == kNormal) {
                        double p0, p1, p2, y0, y1, y2;
                        const int an = rowflag_of(row);
                        if (an >= 0) {
                            p0 = pact_ref(3 * an); p1 = pact_ref(3 * an + 1); p2 = pact_ref(3 * an + 2);
                            y0 = yact_ref(3 * an); y1 = yact_ref(3 * an + 1); y2 = yact_ref(3 * an + 2);
                        } else {
                            VT q0, q1, q2, u0, u1, u2;
                            ld_p(pnew, row, q0, q1, q2);
                            ld_y(row, u0, u1, u2);
                            p0 = q0; p1 = q1; p2 = q2; y0 = u0; y1 = u1; y2 = u2;
                        }
                        double x0, x1, x2;
                        ld_x(row, x0, x1, x2);
                        ld_r(row, r0, r1, r2);
                        x0 += alpha * p0; x1 += alpha * p1; x2 += alpha * p2;
                        r0 -= alpha * y0; r1 -= alpha * y1; r2 -= alpha * y2;
                        st_x(row, x0, x1, x2);
                        st_r(row, r0, r1, r2);
                    } else {
                        ld_r(row, r0, r1, r2);
                    }
                    double t0, t1, t2;
                    dinv_row(row, r0, r1, r2, t0, t1, t2);
                    st_t(tbuf(tc), row, (VT)t0, (VT)t1, (VT)t2);
                    const VT z0 = (VT)(w0 * t0), z1 = (VT)(w0 * t1), z2 = (VT)(w0 * t2);
                    st_z(row, z0, z1, z2);
                    acc_rr += r0 * r0 + r1 * r1 + r2 * r2;
                    acc_rz += r0 * (double)z0 + r1 * (double)z1 + r2 * (double)z2;
                }
                mark(13);
                if (slot == kNormal) {
                    ++it;
                    pc ^= 1;
                }
                if (nterms == 1) compute_zpart();
                else if (schur) compute_part(tbuf(tc), s_to, tpart_half(0) + aidx, nact);
            }
            if (!work) slot = kIdle;
            tail_k0 = (work && fused_slot) ? 2 : 1;
            mark(3);
            const bool rz_here = nterms == 1 || (work && fused_slot && nterms == 2);
            if (!barrier(prm.part_rr, acc_rr, rz_here ? prm.part_rz : nullptr, acc_rz)) return;
            mark(4);
        }
        prev_slot = slot;
        // ---- phases C ----
        tail_active = slot != kIdle;
        ++slot_no;
    }
}

template <class MT, class PT, class VT, int TPR>
cudaError_t launch_t(const PcgParams& prm, int grid, cudaStream_t st, size_t smem) {
    auto fn = pcg_kernel<MT, PT, VT, TPR>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void* args[] = {(void*)&prm};
    e = cudaLaunchCooperativeKernel((void*)fn, dim3(grid), dim3(kThreads), args, smem, st);
    debug_sync("pcg_kernel");
    return e;
}

template <class MT, class PT, class VT, int TPR>
int bps_t(size_t smem) {
    auto fn = pcg_kernel<MT, PT, VT, TPR>;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kThreads, smem);
    return b;
}

}  // namespace

void read_fail_pcg(long long* out) { hsc_read_fail(out); }

size_t pcg_smem_bytes(int vt_doubles, int kmax_all) {
    (void)kmax_all;
    return sizeof(double) * (size_t)(kMaxRank + vt_doubles);
}

cudaError_t launch_pcg(int precision, int tpr, const PcgParams& prm, int grid, size_t smem, cudaStream_t st) {
    count_launch();
#define HSC_PCG_CASE(MT, PT, VT)                                               \
    switch (tpr) {                                                             \
        case 2: return launch_t<MT, PT, VT, 2>(prm, grid, st, smem);           \
        case 8: return launch_t<MT, PT, VT, 8>(prm, grid, st, smem);           \
        default: return launch_t<MT, PT, VT, 4>(prm, grid, st, smem);          \
    }
    if (precision == 0) { HSC_PCG_CASE(double, double, double) }
    if (precision == 1) { HSC_PCG_CASE(float, float, float) }
    HSC_PCG_CASE(float, __nv_bfloat16, float)
#undef HSC_PCG_CASE
}

int pcg_blocks_per_sm(int precision, int tpr, size_t smem) {
#define HSC_BPS_CASE(MT, PT, VT)                                               \
    switch (tpr) {                                                             \
        case 2: return bps_t<MT, PT, VT, 2>(smem);                             \
        case 8: return bps_t<MT, PT, VT, 8>(smem);                             \
        default: return bps_t<MT, PT, VT, 4>(smem);                            \
    }
    if (precision == 0) { HSC_BPS_CASE(double, double, double) }
    if (precision == 1) { HSC_BPS_CASE(float, float, float) }
    HSC_BPS_CASE(float, __nv_bfloat16, float)
#undef HSC_BPS_CASE
}

}  // namespace hsc

// ---------------------------------------------------------------------------
// Self-test of the PCG's grid barrier failure path (failure detection without a
// GPU fault): one cooperative launch in which CTA `absent` never arrives, so
// barrier 0 cannot complete.  CTA 1 waits at most `first_limit` polls, gives
// up, raises the abort flag and sets the counter's top bit; the other CTAs,
// with a much larger limit, must then leave at once and report failure.  Every
// wait is bounded by its poll limit.
// ---------------------------------------------------------------------------
namespace hsc {
namespace {
__global__ void barrier_selftest_kernel(GridBar* gb, int absent, long long first_limit, long long limit, int* status) {
    if (threadIdx.x != 0) return;
    if ((int)blockIdx.x == absent) { status[blockIdx.x] = 2; return; }
    const long long lim = blockIdx.x == 1 ? first_limit : limit;
    status[blockIdx.x] = grid_arrive_wait(gb, gridDim.x, lim, 0) ? 1 : 0;
}
}  // namespace
}  // namespace hsc

extern "C" int hsc_debug_barrier_selftest(int32_t ctas, int32_t absent, int64_t first_limit, int64_t limit,
                                          int32_t* statuses, int32_t* abort_flag, int32_t* where) {
    using namespace hsc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return HSC_ERR_CUDA;
    if (ctas < 2 || ctas > sms || !statuses || first_limit < 1 || limit < first_limit || limit > 100000000)
        return HSC_ERR_INVALID;
    GridBar* gb = nullptr;
    int* st = nullptr;
    if (cudaMalloc(&gb, sizeof(GridBar)) != cudaSuccess) return HSC_ERR_ALLOC;
    if (cudaMalloc(&st, sizeof(int) * ctas) != cudaSuccess) { cudaFree(gb); return HSC_ERR_ALLOC; }
    int rc = HSC_OK;
    GridBar h{};
    if (cudaMemset(gb, 0, sizeof(GridBar)) != cudaSuccess || cudaMemset(st, 0xff, sizeof(int) * ctas) != cudaSuccess) {
        rc = HSC_ERR_CUDA;
    } else {
        long long fl = first_limit, l = limit;
        int ab = absent;
        void* args[] = {&gb, &ab, &fl, &l, &st};
        count_launch();
        if (cudaLaunchCooperativeKernel((void*)barrier_selftest_kernel, dim3(ctas), dim3(32), args, 0, 0) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(statuses, st, sizeof(int) * ctas, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&h, gb, sizeof(GridBar), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = HSC_ERR_CUDA;
    }
    if (abort_flag) *abort_flag = h.abort;
    if (where) *where = h.where;
    cudaFree(gb);
    cudaFree(st);
    return rc;
}

// ---------------------------------------------------------------------------
// z += omega * blockdiag(B) x at the authors' kernel shape (dmv_accumulate_kernel of
// Guo-2026-HSC sparse_linear_solvers/conjugate_gradient_cuda.cuh, exercised by
// reproduction/cuda_original.py with bs 3 and 12).  For bs = 3 the block product is
// the PCG kernel's own dinv_apply over 9 planes d[e * nb + b]; bs = 12 applies the
// same row-major arithmetic to 144 planes.  Test hook: no reference counterpart in
// the solve itself.
// ---------------------------------------------------------------------------
namespace hsc {
namespace {
template <int BS>
__global__ void dmv_accumulate_kernel(int nb, const double* planes, const double* x, double* z, double omega) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    if constexpr (BS == 3) {
        double o0, o1, o2;
        dinv_apply(planes, nb, b, omega, x[3 * b], x[3 * b + 1], x[3 * b + 2], o0, o1, o2);
        z[3 * b] += o0;
        z[3 * b + 1] += o1;
        z[3 * b + 2] += o2;
    } else {
        for (int i = 0; i < BS; ++i) {
            double acc = 0.0;
            for (int j = 0; j < BS; ++j) acc += planes[(size_t)(i * BS + j) * nb + b] * x[BS * b + j];
            z[BS * b + i] += omega * acc;
        }
    }
}
}  // namespace
}  // namespace hsc

extern "C" int hsc_debug_dmv_accumulate(int32_t bs, int32_t nblocks, const double* d_planes, const double* d_x,
                                        double* d_z, double omega, void* stream) {
    using namespace hsc;
    if (nblocks < 0 || (nblocks > 0 && (!d_planes || !d_x || !d_z))) return HSC_ERR_INVALID;
    if (nblocks == 0) return HSC_OK;
    const int grid = (nblocks + 127) / 128;
    cudaStream_t st = (cudaStream_t)stream;
    count_launch();
    if (bs == 3) dmv_accumulate_kernel<3><<<grid, 128, 0, st>>>(nblocks, d_planes, d_x, d_z, omega);
    else if (bs == 12) dmv_accumulate_kernel<12><<<grid, 128, 0, st>>>(nblocks, d_planes, d_x, d_z, omega);
    else return HSC_ERR_INVALID;
    return cudaGetLastError() == cudaSuccess ? HSC_OK : HSC_ERR_CUDA;
}
