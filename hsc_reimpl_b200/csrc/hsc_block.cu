// Block-local Woodbury preconditioner and pipelined Schur PCG (see hsc_block.cuh).
#include <algorithm>
#include <type_traits>

#include "../../include/hsc_c_api.h"
#include "hsc_block.cuh"
#include "hsc_check.cuh"
#include "hsc_setup.cuh"

namespace hsc {

namespace {

// the storage type of Dd^-1: float beside the FP32 planes, double beside FP64 ones.  The
// arithmetic is FP64 throughout: the Woodbury core amplifies any difference between the L that
// built Y and the L the PCG applies, so L must be the same linear map to FP64 rounding.
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

// the 3x3 block (row-major: y_r = sum_c b[3 r + c] x_c) of lane `lane` in a chunk of kChunkVals
// values: planes 0-3 as [lane][4], planes 4-7 as [lane][4], plane 8 as [lane]
template <class MT>
__device__ __forceinline__ void ld_blk(const MT* chunk, int lane, bool global, MT b[9]) {
    if constexpr (std::is_same<MT, float>::value) {
        const float4* c0 = reinterpret_cast<const float4*>(chunk) + lane;
        const float4* c1 = reinterpret_cast<const float4*>(chunk + 128) + lane;
        const float4 q0 = global ? __ldg(c0) : *c0;
        const float4 q1 = global ? __ldg(c1) : *c1;
        b[0] = q0.x; b[1] = q0.y; b[2] = q0.z; b[3] = q0.w;
        b[4] = q1.x; b[5] = q1.y; b[6] = q1.z; b[7] = q1.w;
        b[8] = global ? __ldg(chunk + 256 + lane) : chunk[256 + lane];
    } else {
        const double2* c0 = reinterpret_cast<const double2*>(chunk) + 2 * lane;
        const double2* c1 = reinterpret_cast<const double2*>(chunk + 128) + 2 * lane;
        const double2 q0 = global ? __ldg(c0) : c0[0], q1 = global ? __ldg(c0 + 1) : c0[1];
        const double2 q2 = global ? __ldg(c1) : c1[0], q3 = global ? __ldg(c1 + 1) : c1[1];
        b[0] = q0.x; b[1] = q0.y; b[2] = q1.x; b[3] = q1.y;
        b[4] = q2.x; b[5] = q2.y; b[6] = q3.x; b[7] = q3.y;
        b[8] = global ? __ldg(chunk + 256 + lane) : chunk[256 + lane];
    }
}

// ---------------------------------------------------------------------------
// sliced-ELL values from the BSR planes: one thread per slot (padding slots get zeros)
// ---------------------------------------------------------------------------
template <class MT>
__global__ void block_fill_kernel(const BlockPlan p) {
    const long long nslot = p.nchunk * 32;
    const MT* vals = reinterpret_cast<const MT*>(p.vals);
    MT* out = reinterpret_cast<MT*>(p.sell_vals);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nslot; e += (long long)gridDim.x * blockDim.x) {
        const int src = p.sell_src[e];
        const int lane = (int)(e & 31);
        MT b[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) b[q] = src >= 0 ? vals[(size_t)q * p.nnz + src] : MT(0);
        MT* c = out + (e >> 5) * kChunkVals;
        if constexpr (std::is_same<MT, float>::value) {
            reinterpret_cast<float4*>(c)[lane] = make_float4(b[0], b[1], b[2], b[3]);
            reinterpret_cast<float4*>(c + 128)[lane] = make_float4(b[4], b[5], b[6], b[7]);
        } else {
            reinterpret_cast<double2*>(c)[2 * lane] = make_double2(b[0], b[1]);
            reinterpret_cast<double2*>(c)[2 * lane + 1] = make_double2(b[2], b[3]);
            reinterpret_cast<double2*>(c + 128)[2 * lane] = make_double2(b[4], b[5]);
            reinterpret_cast<double2*>(c + 128)[2 * lane + 1] = make_double2(b[6], b[7]);
        }
        c[256 + lane] = b[8];
    }
}

// ---------------------------------------------------------------------------
// columns of each coupling component: the body of U[:, j]'s first nonzero row
// gives its component (a warp per column, its lanes over 32 rows at a time);
// counting sort into comp_col_ptr / comp_cols (one CTA, kmax <= kMaxRank)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) block_columns_kernel(BlockPlan p) {
    __shared__ int s_cnt[257];
    __shared__ int s_comp[kMaxRank];
    const int k = *p.rank;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int g = threadIdx.x; g <= p.ncomp; g += blockDim.x) s_cnt[g] = 0;
    __syncthreads();
    for (int j = warp; j < p.kmax; j += nwarps) {
        int comp = -1;
        if (j < k) {
            constexpr int kPre = 8;  // the first 256 rows' loads in flight at once
            bool nzr[kPre];
#pragma unroll
            for (int c = 0; c < kPre; ++c) {
                const int i = 32 * c + lane;
                nzr[c] = i < p.qm && p.U[(size_t)j * p.qm + i] != 0.0;
            }
#pragma unroll
            for (int c = 0; c < kPre; ++c) {
                const unsigned nz = __ballot_sync(0xffffffffu, nzr[c]);
                if (comp < 0 && nz) comp = p.comp_of_body[(32 * c + __ffs(nz) - 1) / 12];
            }
            for (int i0 = 32 * kPre; i0 < p.qm && comp < 0; i0 += 32) {
                const int i = i0 + lane;
                const unsigned nz = __ballot_sync(0xffffffffu, i < p.qm && p.U[(size_t)j * p.qm + i] != 0.0);
                if (nz) comp = p.comp_of_body[(i0 + __ffs(nz) - 1) / 12];
            }
        }
        if (lane == 0) {
            s_comp[j] = comp;
            p.comp_of_col[j] = comp;
            if (comp >= 0) atomicAdd(&s_cnt[comp + 1], 1);
        }
    }
    __shared__ int s_sptr[257];
    for (int g = threadIdx.x; g <= p.ncomp; g += blockDim.x) s_sptr[g] = p.comp_slot_ptr[g];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int g = 0; g < p.ncomp; ++g) s_cnt[g + 1] += s_cnt[g];
        for (int g = 0; g <= p.ncomp; ++g) p.comp_col_ptr[g] = s_cnt[g];
        // columns in increasing order inside each component (deterministic)
        for (int j = 0; j < k; ++j) {
            const int comp = s_comp[j];
            if (comp >= 0) p.comp_cols[s_cnt[comp]++] = j;
        }
    } else if (threadIdx.x == 32) {
        // packed partials: column j's contributor slots at col_off[j] ..
        int off = 0;
        for (int j = 0; j < p.kmax; ++j) {
            p.col_off[j] = off;
            const int comp = j < k ? s_comp[j] : -1;
            if (comp >= 0) off += s_sptr[comp + 1] - s_sptr[comp];
        }
        p.col_off[p.kmax] = off;
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
// shared-memory staging of a CTA's part: its slices, the rows' local slot
// counts, the slots' window positions, the value chunks (when staged), the
// Dd^-1 planes, the coupled rows' FP64 diagonal blocks (mixed modes) and (for
// the operator) the window node ids
// ---------------------------------------------------------------------------
template <class MT>
struct Part {
    int rb, re, R, ns, nch, wn0, nwin, wown, ab, ae, na;
    const int4* meta;                  // per slice: first chunk (from the CTA's first), chunks, local chunks
    const unsigned short* nloc;        // per row: slots holding its diagonal and local blocks
    const unsigned short* lc;          // per slot: window position
    const MT* val;                     // chunks (shared or global)
    const typename BlkDinv<MT>::T* dinv;  // planes, stride R
    const int* aflag;                  // per row: its coupled node among the CTA's, or -1
    const double* dact;                // 9 per coupled node of the CTA (mixed modes), else null
    int* wn;
};

template <class MT>
__device__ Part<MT> stage_part(const BlockPlan& p, int cta, unsigned char* sm, bool window) {
    using DT = typename BlkDinv<MT>::T;
    Part<MT> s;
    s.rb = p.cta_row[2 * cta];
    s.re = p.cta_row[2 * cta + 1];
    s.R = s.re - s.rb;
    const int sl0 = p.cta_slice[cta];
    s.ns = p.cta_slice[cta + 1] - sl0;
    const long long ch0 = p.cta_chunk[cta];
    s.nch = p.cta_chunk[cta + 1] - (int)ch0;
    s.wn0 = p.win_off[cta];
    s.nwin = p.win_off[cta + 1] - s.wn0;
    s.wown = p.win_own[cta];
    s.ab = p.cta_act[2 * cta];
    s.ae = p.cta_act[2 * cta + 1];
    s.na = s.ae - s.ab;
    int4* meta = reinterpret_cast<int4*>(sm + p.off_meta);
    unsigned short* nloc = reinterpret_cast<unsigned short*>(sm + p.off_nloc);
    unsigned short* lc = reinterpret_cast<unsigned short*>(sm + p.off_lc);
    DT* sd = reinterpret_cast<DT*>(sm + p.off_dinv);
    s.wn = reinterpret_cast<int*>(sm + p.off_wn);
    const DT* dinv = reinterpret_cast<const DT*>(p.dinv);
    const MT* vals = reinterpret_cast<const MT*>(p.sell_vals) + ch0 * kChunkVals;
    for (int e = threadIdx.x; e < s.ns; e += blockDim.x) meta[e] = p.sell_slice[sl0 + e];
    for (int e = threadIdx.x; e < s.R; e += blockDim.x) nloc[e] = p.sell_nloc[s.rb + e];
    {
        const uint4* src = reinterpret_cast<const uint4*>(p.sell_lc + ch0 * 32);  // 64 B per chunk
        uint4* dst = reinterpret_cast<uint4*>(lc);
        for (int e = threadIdx.x; e < 4 * s.nch; e += blockDim.x) dst[e] = __ldg(src + e);
    }
    if (window)
        for (int e = threadIdx.x; e < s.nwin; e += blockDim.x) s.wn[e] = p.win_nodes[s.wn0 + e];
    for (int e = threadIdx.x; e < 9 * s.R; e += blockDim.x) {
        const int pl = e / s.R, lr = e - pl * s.R;
        sd[e] = dinv[(size_t)pl * p.n + s.rb + lr];
    }
    int* aflag = reinterpret_cast<int*>(sm + p.off_aflag);
    for (int e = threadIdx.x; e < s.R; e += blockDim.x) {
        const int an = p.rowflag[s.rb + e];
        aflag[e] = an >= 0 ? an - s.ab / 3 : -1;
    }
    double* sdact = reinterpret_cast<double*>(sm + p.off_dact);
    if (p.dact)
        for (int e = threadIdx.x; e < 3 * s.na; e += blockDim.x) sdact[e] = p.dact[(size_t)3 * s.ab + e];
    s.aflag = aflag;
    s.dact = p.dact ? sdact : nullptr;
    if (p.stage_vals) {
        const int4* src = reinterpret_cast<const int4*>(vals);
        int4* dst = reinterpret_cast<int4*>(sm + p.off_val);
        const int n16 = (int)(s.nch * kChunkVals * sizeof(MT) / 16);
        for (int e = threadIdx.x; e < n16; e += blockDim.x) dst[e] = __ldg(src + e);
        s.val = reinterpret_cast<const MT*>(sm + p.off_val);
    } else {
        s.val = vals;
    }
    s.meta = meta;
    s.nloc = nloc;
    s.lc = lc;
    s.dinv = sd;
    __syncthreads();
    return s;
}

__device__ __forceinline__ double poly_weight(const BlockPlan& p, int k) { return p.wdev ? p.wdev[k] : p.w[k]; }

// z_c = L v_c for the NB vectors c of a batch, over the CTA's rows:
//   t_0 = w Dd^-1 v,  t_k = (1 - w) t_{k-1} - w Dd^-1 (O t_{k-1}),  z = sum_k w_k t_k,
// O the blocks between two different rows of the part (Dd^-1 D_loc = I + Dd^-1 O), so each
// term is one pass over the rows' local slots and no grid barrier.  In the mixed modes a
// coupled row keeps t_k = t_{k-1} - w Dd^-1 (Dc t_{k-1} + O t_{k-1}) with its FP64 diagonal block
// Dc: D - V C V^T cancels most of Dc there, and a Dd^-1 rounded to FP32 is not Dc's inverse
// closely enough to drop the product (about a third more PCG iterations on a vehicle).
// v, z, t, u: NB x 3R doubles (3 per row; stride ld).  Rows are 24 bytes apart, so the gathers
// of a warp spread over the banks.  The slot loop has no branch (a slot that is not a local
// block reads row 0 and adds zero), so consecutive slots' loads overlap.  Ends synchronised;
// z holds the result.
template <class MT, int NB>
__device__ void part_poly(const BlockPlan& p, const Part<MT>& s, const double* v, double* z, double* t, double* u,
                          int ld) {
    using DT = typename BlkDinv<MT>::T;
    const bool gv = !p.stage_vals;
    const double om = p.omega, om1 = 1.0 - p.omega;
    const double w0 = poly_weight(p, 0);
    for (int e = threadIdx.x; e < NB * s.R; e += blockDim.x) {
        const int c = e / s.R, lr = e - c * s.R;
        const size_t o = (size_t)c * ld + 3 * lr;
        double o0, o1, o2;
        blk_dinv<DT>(s.dinv, s.R, lr, om, v[o], v[o + 1], v[o + 2], o0, o1, o2);
        t[o] = o0; t[o + 1] = o1; t[o + 2] = o2;
        z[o] = w0 * o0; z[o + 1] = w0 * o1; z[o + 2] = w0 * o2;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, h = lane & 1;
    double* tc = t;
    double* tn = u;
    for (int k = 1; k < p.nterms; ++k) {
        const double wk = poly_weight(p, k);
        for (int sl = warp; sl < s.ns; sl += kWarps) {
            const int4 m = s.meta[sl];
            const int lr = kSliceRows * sl + (lane >> 1);
            const bool ok = lr < s.R;
            const int nl = ok ? (int)s.nloc[lr] : 0;
            double a[NB][3];
#pragma unroll
            for (int c = 0; c < NB; ++c) a[c][0] = a[c][1] = a[c][2] = 0.0;
#pragma unroll 2
            for (int cc = 0; cc < m.z; ++cc) {
                const int j = 2 * cc + h;
                const bool use = j >= 1 && j < nl;  // slot 0 is the diagonal block
                const int ch = m.x + cc;
                const int ol = use ? (int)s.lc[ch * 32 + lane] - s.wown : 0;
                MT b[9];
                ld_blk<MT>(s.val + (size_t)ch * kChunkVals, lane, gv, b);
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    const double* xc = tc + (size_t)c * ld + 3 * ol;
                    const double x0 = use ? xc[0] : 0.0, x1 = use ? xc[1] : 0.0, x2 = use ? xc[2] : 0.0;
                    a[c][0] += (double)b[0] * x0 + (double)b[1] * x1 + (double)b[2] * x2;
                    a[c][1] += (double)b[3] * x0 + (double)b[4] * x1 + (double)b[5] * x2;
                    a[c][2] += (double)b[6] * x0 + (double)b[7] * x1 + (double)b[8] * x2;
                }
            }
#pragma unroll
            for (int c = 0; c < NB; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d) a[c][d] += __shfl_xor_sync(0xffffffffu, a[c][d], 1);
            if (ok && h == 0) {
                const int an = s.dact ? s.aflag[lr] : -1;
#pragma unroll
                for (int c = 0; c < NB; ++c) {
                    const size_t o = (size_t)c * ld + 3 * lr;
                    const double c0 = tc[o], c1 = tc[o + 1], c2 = tc[o + 2];
                    double f = om1, e0, e1, e2;
                    if (an >= 0) {
                        const double* d = s.dact + 9 * an;
                        a[c][0] += d[0] * c0 + d[1] * c1 + d[2] * c2;
                        a[c][1] += d[3] * c0 + d[4] * c1 + d[5] * c2;
                        a[c][2] += d[6] * c0 + d[7] * c1 + d[8] * c2;
                        f = 1.0;
                    }
                    blk_dinv<DT>(s.dinv, s.R, lr, om, a[c][0], a[c][1], a[c][2], e0, e1, e2);
                    const double n0 = f * c0 - e0, n1 = f * c1 - e1, n2 = f * c2 - e2;
                    tn[o] = n0; tn[o + 1] = n1; tn[o + 2] = n2;
                    z[o] += wk * n0; z[o + 1] += wk * n1; z[o + 2] += wk * n2;
                }
            }
        }
        __syncthreads();
        double* tmp = tc; tc = tn; tn = tmp;
    }
}

// out = D m over the CTA's rows: every slot of every row (padding slots, and the slots of the
// rows past R, hold zeros and a valid window position), m from the staged window (3 doubles per
// window node), FP64; in the mixed modes the coupled rows' diagonal blocks come from the staged
// FP64 copies and `own`.
template <class MT>
__device__ void part_op(const Part<MT>& s, bool gv, const double* win, const double* own, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int sl = warp; sl < s.ns; sl += kWarps) {
        const int4 m = s.meta[sl];
        const int lr = kSliceRows * sl + (lane >> 1);
        const bool ok = lr < s.R;
        double a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 2
        for (int cc = 0; cc < m.y; ++cc) {
            const int ch = m.x + cc;
            const int w = s.lc[ch * 32 + lane];
            MT b[9];
            ld_blk<MT>(s.val + (size_t)ch * kChunkVals, lane, gv, b);
            const double x0 = win[3 * w], x1 = win[3 * w + 1], x2 = win[3 * w + 2];
            a0 += (double)b[0] * x0 + (double)b[1] * x1 + (double)b[2] * x2;
            a1 += (double)b[3] * x0 + (double)b[4] * x1 + (double)b[5] * x2;
            a2 += (double)b[6] * x0 + (double)b[7] * x1 + (double)b[8] * x2;
        }
        a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 1);
        if (ok && (lane & 1) == 0) {
            if (s.dact) {
                const int an = s.aflag[lr];
                if (an >= 0) {
                    const double* d = s.dact + 9 * an;
                    const double x0 = own[3 * lr], x1 = own[3 * lr + 1], x2 = own[3 * lr + 2];
                    a0 += d[0] * x0 + d[1] * x1 + d[2] * x2;
                    a1 += d[3] * x0 + d[4] * x1 + d[5] * x2;
                    a2 += d[6] * x0 + d[7] * x1 + d[8] * x2;
                }
            }
            out[3 * lr] = a0; out[3 * lr + 1] = a1; out[3 * lr + 2] = a2;
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-balanced passes over a CTA's chunks (the PCG kernel).  The chunks of the
// CTA's slices form one sequence (the polynomial takes each slice's leading
// local chunks, the operator all of them); warp w takes the positions
// [T w / W, T (w + 1) / W) of the T in the sequence, so no warp waits on the
// widest slice.  A warp's run through one slice is a segment: it leaves the 16
// rows' partial sums in shared memory, and a second pass (a thread per row) adds
// the segments of the row's slice in sequence order, so sums are deterministic.
// ---------------------------------------------------------------------------
constexpr int kMaxSlices = (kBlockMaxRows + kSliceRows - 1) / kSliceRows;
constexpr int kMaxSegs = kWarps + kMaxSlices;

struct WarpPlan {
    short fs[kWarps];            // first slice of the warp's run
    short fc[kWarps];            // its first chunk inside that slice
    short nc[kWarps];            // chunks in the run
    short seg0[kWarps];          // the run's first segment
    short sg[kMaxSlices + 1];    // segments of slice s: sg[s] .. sg[s + 1]
};

// a slice's chunk range in a pass: local slots [0, z), remote slots [w, y)
enum { kRunLocal = 0, kRunRemote = 1 };
__device__ __forceinline__ int run_base(const int4& m, int mode) { return mode == kRunRemote ? m.w : 0; }
__device__ __forceinline__ int run_len(const int4& m, int mode) { return mode == kRunRemote ? m.y - m.w : m.z; }

// one thread: the plan of a pass over the slices' ranges (mode kRunLocal or kRunRemote) split over
// warps [0, nw); the warps from nw on get empty runs
__device__ void make_warp_plan(const int4* meta, int ns, int mode, WarpPlan& P, int nw = kWarps) {
    int tot = 0;
    for (int s = 0; s < ns; ++s) tot += run_len(meta[s], mode);
    int s = 0, off = 0, seg = 0;
    for (int sl = 0; sl <= ns; ++sl) P.sg[sl] = -1;
    for (int w = 0; w < kWarps; ++w) {
        const int ww = min(w, nw);
        const int p0 = (int)((long long)tot * ww / nw), p1 = w < nw ? (int)((long long)tot * (ww + 1) / nw) : p0;
        while (s < ns && off + run_len(meta[s], mode) <= p0) { off += run_len(meta[s], mode); ++s; }
        P.fs[w] = (short)s;
        P.fc[w] = (short)(p0 - off);
        P.nc[w] = (short)(p1 - p0);
        P.seg0[w] = (short)seg;
        int ss = s, o = off, q = p0;
        while (q < p1) {  // one segment per slice the run touches
            const int len = run_len(meta[ss], mode);
            if (P.sg[ss] < 0) P.sg[ss] = (short)seg;
            ++seg;
            q = min(p1, o + len);
            if (q < p1) { o += len; ++ss; }
        }
    }
    P.sg[ns] = (short)seg;
    for (int sl = ns - 1; sl >= 0; --sl)
        if (P.sg[sl] < 0) P.sg[sl] = P.sg[sl + 1];
}

// phase 1 of a balanced pass: warp `warp` walks its run and leaves, per segment g, the 16 rows'
// sums of the slots `pick` admits times x (x_of(lane, window position) gives the 3 entries)
template <class MT, class Pick, class XOf>
__device__ __forceinline__ void run_segments(const Part<MT>& s, const WarpPlan& P, int mode, bool gv, double* scratch,
                                             Pick pick, XOf x_of) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, h = lane & 1;
    int sl = P.fs[warp], c = P.fc[warp], left = P.nc[warp], g = P.seg0[warp];
    while (left > 0) {
        const int4 m0 = s.meta[sl];
        const int base = run_base(m0, mode);
        const int4 m = make_int4(m0.x + base, 0, 0, 0);   // chunk cc of the run is chunk base + cc of the slice
        const int len = run_len(m0, mode);
        const int cend = min(len, c + left);
        const int lr = kSliceRows * sl + (lane >> 1);
        const bool ok = lr < s.R;
        const int nl = ok ? (int)s.nloc[lr] : 0;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll 2
        for (int cc = c; cc < cend; ++cc) {
            const int j = 2 * (base + cc) + h;
            const bool use = pick(j, nl);
            const int ch = m.x + cc;
            const int w = s.lc[ch * 32 + lane];
            MT b[9];
            ld_blk<MT>(s.val + (size_t)ch * kChunkVals, lane, gv, b);
            double x0, x1, x2;
            x_of(use, w, x0, x1, x2);
            a0 += (double)b[0] * x0 + (double)b[1] * x1 + (double)b[2] * x2;
            a1 += (double)b[3] * x0 + (double)b[4] * x1 + (double)b[5] * x2;
            a2 += (double)b[6] * x0 + (double)b[7] * x1 + (double)b[8] * x2;
        }
        a0 += __shfl_xor_sync(0xffffffffu, a0, 1);
        a1 += __shfl_xor_sync(0xffffffffu, a1, 1);
        a2 += __shfl_xor_sync(0xffffffffu, a2, 1);
        if (h == 0) {
            double* o = scratch + ((size_t)g * kSliceRows + (lane >> 1)) * 3;
            o[0] = a0; o[1] = a1; o[2] = a2;
        }
        left -= cend - c;
        c = 0;
        ++sl;
        ++g;
    }
}

// the sum of row lr's segments
__device__ __forceinline__ void seg_sum(const WarpPlan& P, const double* scratch, int lr, double& y0, double& y1,
                                        double& y2) {
    const int sl = lr / kSliceRows, r = lr - sl * kSliceRows;
    y0 = y1 = y2 = 0.0;
    for (int g = P.sg[sl]; g < P.sg[sl + 1]; ++g) {
        const double* o = scratch + ((size_t)g * kSliceRows + r) * 3;
        y0 += o[0]; y1 += o[1]; y2 += o[2];
    }
}

// asynchronous 8-byte copy global -> shared (no register holds the value), and the wait for all of
// the thread's copies
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// the thread of the last warp, which owns no row (R <= kBlockMaxRows) and so idles through every
// row loop: it signals grid barriers and looks at their counters while the other warps work
constexpr int kIdleThread = kThreads - 32;
static_assert(kBlockMaxRows <= kIdleThread, "the last warp must own no row");

// z = L v over the CTA's rows, warp-balanced (the polynomial of part_poly for one vector; v, z,
// t, u: 3 per row).  Ends synchronised.  hook(0) runs once every thread's earlier writes are
// ordered before it (after the first product's partial sums, or after the first term when there
// is no product), hook(1) while the last product's rows are updated; both on every thread, for
// kIdleThread to act on.
template <class MT, class Hook>
__device__ void part_poly_bal(const BlockPlan& p, const Part<MT>& s, const WarpPlan& P, double* scratch,
                              const double* v, double* z, double* t, double* u, Hook hook) {
    using DT = typename BlkDinv<MT>::T;
    const bool gv = !p.stage_vals;
    const double om = p.omega, om1 = 1.0 - p.omega;
    const double w0 = poly_weight(p, 0);
    for (int lr = threadIdx.x; lr < s.R; lr += blockDim.x) {
        double o0, o1, o2;
        blk_dinv<DT>(s.dinv, s.R, lr, om, v[3 * lr], v[3 * lr + 1], v[3 * lr + 2], o0, o1, o2);
        t[3 * lr] = o0; t[3 * lr + 1] = o1; t[3 * lr + 2] = o2;
        z[3 * lr] = w0 * o0; z[3 * lr + 1] = w0 * o1; z[3 * lr + 2] = w0 * o2;
    }
    __syncthreads();
    if (p.nterms <= 1) hook(0);
    double* tc = t;
    double* tn = u;
    for (int k = 1; k < p.nterms; ++k) {
        const double wk = poly_weight(p, k);
        const double* xs = tc;
        run_segments<MT>(
            s, P, kRunLocal, gv, scratch, [](int j, int nl) { return j >= 1 && j < nl; },  // slot 0: the diagonal
            [&](bool use, int w, double& x0, double& x1, double& x2) {
                const int ol = use ? w - s.wown : 0;
                x0 = use ? xs[3 * ol] : 0.0; x1 = use ? xs[3 * ol + 1] : 0.0; x2 = use ? xs[3 * ol + 2] : 0.0;
            });
        __syncthreads();
        if (k == 1) hook(0);
        if (k == p.nterms - 1) hook(1);
        for (int lr = threadIdx.x; lr < s.R; lr += blockDim.x) {
            double y0, y1, y2, e0, e1, e2;
            seg_sum(P, scratch, lr, y0, y1, y2);
            const double c0 = tc[3 * lr], c1 = tc[3 * lr + 1], c2 = tc[3 * lr + 2];
            double f = om1;
            const int an = s.dact ? s.aflag[lr] : -1;
            if (an >= 0) {
                const double* d = s.dact + 9 * an;
                y0 += d[0] * c0 + d[1] * c1 + d[2] * c2;
                y1 += d[3] * c0 + d[4] * c1 + d[5] * c2;
                y2 += d[6] * c0 + d[7] * c1 + d[8] * c2;
                f = 1.0;
            }
            blk_dinv<DT>(s.dinv, s.R, lr, om, y0, y1, y2, e0, e1, e2);
            const double n0 = f * c0 - e0, n1 = f * c1 - e1, n2 = f * c2 - e2;
            tn[3 * lr] = n0; tn[3 * lr + 1] = n1; tn[3 * lr + 2] = n2;
            z[3 * lr] += wk * n0; z[3 * lr + 1] += wk * n1; z[3 * lr + 2] += wk * n2;
        }
        __syncthreads();
        double* tmp = tc; tc = tn; tn = tmp;
    }
}

// out = (D m) restricted to the blocks whose column is a row of the part (the diagonal included),
// warp-balanced, m from the part's own rows; the coupled rows' FP64 diagonal blocks in the mixed
// modes.  Needs no other CTA's data.  Ends synchronised.
template <class MT>
__device__ void part_op_local(const Part<MT>& s, const WarpPlan& P, double* scratch, bool gv, const double* own,
                              double* out) {
    run_segments<MT>(
        s, P, kRunLocal, gv, scratch, [](int j, int nl) { return j < nl; },
        [&](bool use, int w, double& x0, double& x1, double& x2) {
            const int ol = use ? w - s.wown : 0;
            x0 = use ? own[3 * ol] : 0.0; x1 = use ? own[3 * ol + 1] : 0.0; x2 = use ? own[3 * ol + 2] : 0.0;
        });
    __syncthreads();
    for (int lr = threadIdx.x; lr < s.R; lr += blockDim.x) {
        double a0, a1, a2;
        seg_sum(P, scratch, lr, a0, a1, a2);
        if (s.dact) {
            const int an = s.aflag[lr];
            if (an >= 0) {
                const double* d = s.dact + 9 * an;
                const double x0 = own[3 * lr], x1 = own[3 * lr + 1], x2 = own[3 * lr + 2];
                a0 += d[0] * x0 + d[1] * x1 + d[2] * x2;
                a1 += d[3] * x0 + d[4] * x1 + d[5] * x2;
                a2 += d[6] * x0 + d[7] * x1 + d[8] * x2;
            }
        }
        out[3 * lr] = a0; out[3 * lr + 1] = a1; out[3 * lr + 2] = a2;
    }
    __syncthreads();
}

// out += the remaining blocks of D m (columns outside the part), warp-balanced, m from the staged
// window (3 doubles per window node).  Ends synchronised.
template <class MT>
__device__ void part_op_remote(const Part<MT>& s, const WarpPlan& P, double* scratch, bool gv, const double* win,
                               double* out) {
    run_segments<MT>(
        s, P, kRunRemote, gv, scratch, [](int j, int nl) { return j >= nl; },
        [&](bool use, int w, double& x0, double& x1, double& x2) {
            x0 = use ? win[3 * w] : 0.0; x1 = use ? win[3 * w + 1] : 0.0; x2 = use ? win[3 * w + 2] : 0.0;
        });
    __syncthreads();
    for (int lr = threadIdx.x; lr < s.R; lr += blockDim.x) {
        double a0, a1, a2;
        seg_sum(P, scratch, lr, a0, a1, a2);
        out[3 * lr] += a0; out[3 * lr + 1] += a1; out[3 * lr + 2] += a2;
    }
    __syncthreads();
}

constexpr int kYBatch = 4;  // columns per pass of the Y kernel

// the V^T Y partial kernel's shared memory: the column list and slots, then V's and Y's rows
__host__ __device__ inline size_t gpart_stage_offset(int kmax) { return ((size_t)8 * kmax + 15) / 16 * 16; }
__host__ __device__ inline size_t gpart_smem_bytes(int kmax, int NA, int NCOL) {
    return gpart_stage_offset(kmax) + sizeof(double) * 2 * (size_t)NA * NCOL;
}

// doubles of the Y kernel's vector region: the batch's inputs and the polynomial's three
// vectors, 3R per column each
__host__ __device__ inline size_t y_region_doubles(int R) { return (size_t)4 * kYBatch * 3 * R; }

// ---------------------------------------------------------------------------
// Y = L V on each part: CTA (part, b) takes columns [4 b, 4 b + 4) of the part's
// column list (the columns of the components in the part), so the batches of a
// part run side by side; it writes Y (FP32, node-padded), Y at the coupled dofs
// (FP32-rounded; the rest of Yact is zeroed before the launch) and the part's
// compact rows of V for its columns
// ---------------------------------------------------------------------------
template <class MT>
__global__ void __launch_bounds__(kThreads, 1) block_y_kernel(const BlockPlan p_arg) {
    using AT = double;
    __shared__ __align__(16) unsigned char s_p_raw[sizeof(BlockPlan)];
    BlockPlan& p = *reinterpret_cast<BlockPlan*>(s_p_raw);
    if (threadIdx.x == 0) p = p_arg;
    __syncthreads();
    extern __shared__ __align__(16) unsigned char sm[];
    const int cta = blockIdx.x;
    constexpr int NB = kYBatch;
    const int q0 = NB * blockIdx.y;
    int* s_cols = reinterpret_cast<int*>(sm + p.off_cols);
    int* s_slot = s_cols + p.kmax;
    const int ncols = build_cols(p, cta, s_cols, s_slot);
    if (q0 >= ncols) return;  // uniform in the CTA
    const Part<MT> s = stage_part<MT>(p, cta, sm, false);
    double* vec = reinterpret_cast<double*>(sm + p.off_vec);
    const int R3 = 3 * p.R;
    double* v = vec;                                   // NB x 3R
    AT* z = reinterpret_cast<AT*>(vec + NB * R3);      // NB x 3R each
    AT* t = z + NB * R3;
    AT* u = t + NB * R3;
    int* s_act = reinterpret_cast<int*>(sm + p.off_act);
    for (int e = threadIdx.x; e < s.na; e += blockDim.x) s_act[e] = p.actp[s.ab + e] - 3 * s.rb;
    for (int e = threadIdx.x; e < NB * R3; e += blockDim.x) v[e] = 0.0;
    __syncthreads();
    for (int e = threadIdx.x; e < NB * s.na; e += blockDim.x) {
        const int c = e / s.na, il = e - c * s.na;
        if (q0 + c < ncols) v[(size_t)c * R3 + s_act[il]] = p.V[(size_t)s_cols[q0 + c] * p.a + p.actperm[s.ab + il]];
    }
    __syncthreads();
    part_poly<MT, NB>(p, s, v, z, t, u, R3);
    // the PCG applies the FP32 copy of Y; the Woodbury core is built from the same rounded values
    for (int e = threadIdx.x; e < NB * s.R; e += blockDim.x) {
        const int c = e / s.R, lr = e - c * s.R;
        if (q0 + c >= ncols) continue;
        const AT* zr = z + (size_t)c * R3 + 3 * lr;
        float* Yj = p.Y + (size_t)s_cols[q0 + c] * 4 * p.n;
        reinterpret_cast<float4*>(Yj)[s.rb + lr] = make_float4((float)zr[0], (float)zr[1], (float)zr[2], 0.f);
    }
    double* Vc = p.Vc + (size_t)p.kmax * s.ab;  // the part's coupled rows of V, compact: [list position q][dof]
    for (int e = threadIdx.x; e < NB * s.na; e += blockDim.x) {
        const int c = e / s.na, il = e - c * s.na;
        if (q0 + c < ncols) {
            const int j = s_cols[q0 + c];
            p.Yact[(size_t)j * p.a + s.ab + il] = (double)(float)z[(size_t)c * R3 + s_act[il]];
            Vc[(size_t)(q0 + c) * s.na + il] = p.V[(size_t)j * p.a + p.actperm[s.ab + il]];
        }
    }
}

// the partial G_c[j][l] = sum over a coupled part's own coupled dofs of V[., j] Yact[., l] (dense
// kmax^2, zero outside its columns).  The part's rows of V ([q][dof]) and of Y ([dof][q]) are staged
// in shared memory when they fit: a warp takes a row q_a, its lanes the columns q_b, and walks the dofs.
__global__ void __launch_bounds__(kThreads, 1) block_gpart_kernel(const BlockPlan p_arg) {
    __shared__ __align__(16) unsigned char s_p_raw[sizeof(BlockPlan)];
    BlockPlan& p = *reinterpret_cast<BlockPlan*>(s_p_raw);
    if (threadIdx.x == 0) p = p_arg;
    __syncthreads();
    const int cta = blockIdx.x;
    const int aidx = p.cta_aidx[cta];
    if (aidx < 0) return;  // uniform in the CTA
    extern __shared__ __align__(16) unsigned char sm[];
    int* s_cols = reinterpret_cast<int*>(sm);  // layout: column list and slots (2 kmax ints), then the staging
    int* s_slot = s_cols + p.kmax;
    const int ncols = build_cols(p, cta, s_cols, s_slot);
    const int k = *p.rank;
    const int ab = p.cta_act[2 * cta], na = p.cta_act[2 * cta + 1] - ab;
    const double* Vc = p.Vc + (size_t)p.kmax * ab;
    double* Gc = p.pG + (size_t)aidx * p.kmax * p.kmax;
    for (int e = threadIdx.x; e < p.kmax * p.kmax; e += blockDim.x) Gc[e] = 0.0;
    double* vec = reinterpret_cast<double*>(sm + gpart_stage_offset(p.kmax));
    const bool staged = p.gpart_staged && ncols <= p.NCOL;
    double* Vs = vec;
    double* Ys = vec + (size_t)na * ncols;
    if (staged)
        for (int e = threadIdx.x; e < ncols * na; e += blockDim.x) {
            const int q = e / na, il = e - q * na;
            Vs[e] = Vc[e];
            Ys[(size_t)il * ncols + q] = p.Yact[(size_t)s_cols[q] * p.a + ab + il];
        }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int qa = warp; qa < ncols; qa += kWarps)
        for (int qb = lane; qb < ncols; qb += 32) {
            const int j = s_cols[qa], l = s_cols[qb];
            double acc = 0.0;
            if (staged) {
                for (int il = 0; il < na; ++il) acc += Vs[(size_t)qa * na + il] * Ys[(size_t)il * ncols + qb];
            } else {
                for (int il = 0; il < na; ++il) acc += Vc[(size_t)qa * na + il] * p.Yact[(size_t)l * p.a + ab + il];
            }
            if (j < k && l < k) Gc[(size_t)j * p.kmax + l] = acc;
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
//   phase 1: partials of Y^T v and of the dots (r,u) (w,u) (r,r), then
//            mt = L v (local)
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
//
// Each thread owns dofs e = tid + kThreads i (i < kDofs) of the CTA's rows and
// keeps x, r, u, p, s, q, z of them in registers; w, m and n, which other
// threads read, live in shared memory.  The rows of K and C for the CTA's
// columns (at most 32 columns of a rank of at most 128) live in registers too.
// ---------------------------------------------------------------------------
enum { kPassStart = 0, kPassNormal = 1 };
constexpr int kDofs = 2;      // 3 R <= kDofs * kThreads  (R <= kBlockMaxRows)
constexpr int kRegCols = 2;   // K and C rows held per warp
constexpr int kRegK = 4;      // 32-wide strips of a K / C row per lane

template <class MT>
__global__ void __launch_bounds__(kThreads, 1) block_pcg_kernel(const BlockPlan p_arg) {
    using AT = double;
    __shared__ __align__(16) unsigned char s_p_raw[sizeof(BlockPlan)];
    BlockPlan& p = *reinterpret_cast<BlockPlan*>(s_p_raw);
    if (threadIdx.x == 0) p = p_arg;
    __syncthreads();
    extern __shared__ __align__(16) unsigned char sm[];
    const int cta = blockIdx.x;
    const unsigned int G = gridDim.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Part<MT> sl = stage_part<MT>(p, cta, sm, true);
    const bool gv = !p.stage_vals;
    const int R = sl.R, R3 = 3 * R, ld = 3 * p.R;
    double* vec = reinterpret_cast<double*>(sm + p.off_vec);
    AT* Pz = vec;                // L v
    double* Wb = vec + ld;       // w (r on a (re)start): the preconditioner's input
    double* Mm = vec + 2 * ld;   // m (x during a true-residual check)
    double* Nn = vec + 3 * ld;   // n = S m
    double* Zv = vec + 4 * ld;   // the recurrences' z, q, s, p
    double* Qv = vec + 5 * ld;
    double* Sv = vec + 6 * ld;
    double* Pv = vec + 7 * ld;
    double* win = reinterpret_cast<double*>(sm + p.off_win);   // 3 per window node
    // the polynomial's two scratch vectors: the window and n, neither live while it runs
    AT* Pt = win;
    AT* Pu = Nn;
    int* s_act = reinterpret_cast<int*>(sm + p.off_act);       // own coupled dofs, local (3 lr + d)
    int* s_cols = reinterpret_cast<int*>(sm + p.off_cols);
    int* s_slot = s_cols + p.kmax;
    int* s_srng = reinterpret_cast<int*>(sm + p.off_srng);     // per column j < k: its packed partials
    double* s_sv = reinterpret_cast<double*>(sm + p.off_kv);  // Y^T v sums (kmax)
    double* s_vt = s_sv + p.kmax;                             // V^T m sums (kmax)
    double* s_c = s_vt + p.kmax;                              // K s on the CTA's columns (by list position)
    double* s_t = s_c + p.kmax;                               // C vt on the CTA's columns
    double* s_red = reinterpret_cast<double*>(sm + p.off_red);// kWarps x 4 scratch
    __shared__ double s_dot[4];
    __shared__ int s_ok;
    // warp runs over the local slots (polynomial), the same over all warps but the last (the local
    // operator blocks, while the last warp signals the barrier) and over the rest
    __shared__ WarpPlan s_plan_loc, s_plan_op, s_plan_rem;
    __shared__ unsigned int s_pre;  // the barrier counter as kIdleThread saw it during the polynomial (0: not looked)
    double* scr = reinterpret_cast<double*>(sm + p.off_scr);   // segment partial sums
    if (threadIdx.x == 0) make_warp_plan(sl.meta, sl.ns, kRunLocal, s_plan_loc);
    if (threadIdx.x == 32) make_warp_plan(sl.meta, sl.ns, kRunRemote, s_plan_rem);
    if (threadIdx.x == 64) make_warp_plan(sl.meta, sl.ns, kRunLocal, s_plan_op, kWarps - 1);
    if (threadIdx.x == 0) s_pre = 0u;
    for (int e = threadIdx.x; e < sl.na; e += blockDim.x) s_act[e] = p.actp[sl.ab + e] - 3 * sl.rb;
    const int ncols = build_cols(p, cta, s_cols, s_slot);  // synchronises: s_act is complete
    const int k = *p.rank;
    // s_slot[q] becomes the position of the CTA's partial for column s_cols[q] in the packed arrays
    for (int q = threadIdx.x; q < ncols; q += blockDim.x) {
        const int j = s_cols[q], g = p.comp_of_col[j];
        s_slot[q] = p.col_off[j] + s_slot[q] - p.comp_slot_ptr[g];
    }
    for (int j = threadIdx.x; j < k; j += blockDim.x) {
        const int g = p.comp_of_col[j];
        s_srng[2 * j] = p.col_off[j];
        s_srng[2 * j + 1] = g >= 0 ? p.col_off[j + 1] : p.col_off[j];
    }
    int epoch = 0;
    // the CTA's first nyc Y columns are staged (3R floats each, after its value chunks), the rest
    // read from L2
    const int nyc = min(ncols, p.cta_yc[2 * cta + 1]);
    if (nyc > 0) {
        float* yc = reinterpret_cast<float*>(sm + p.cta_yc[2 * cta]);
        for (int e = threadIdx.x; e < nyc * R; e += blockDim.x) {
            const int q = e / R, lr = e - q * R;
            const float4 y = reinterpret_cast<const float4*>(p.Y + (size_t)s_cols[q] * 4 * p.n)[sl.rb + lr];
            float* o = yc + (size_t)q * R3 + 3 * lr;
            o[0] = y.x; o[1] = y.y; o[2] = y.z;
        }
    }
    // the rows of K and C for the CTA's columns: column q = warp + kWarps c, entries l = lane + 32 i
    const bool kreg = ncols <= kRegCols * kWarps && k <= 32 * kRegK;
    double kr[kRegCols][kRegK], cr[kRegCols][kRegK];
#pragma unroll
    for (int c = 0; c < kRegCols; ++c)
#pragma unroll
        for (int i = 0; i < kRegK; ++i) {
            const int q = warp + kWarps * c, l = lane + 32 * i;
            const bool in = kreg && q < ncols && l < k;
            kr[c][i] = in ? p.K[(size_t)s_cols[q] * p.kmax + l] : 0.0;
            cr[c][i] = in ? p.C[(size_t)s_cols[q] * p.kmax + l] : 0.0;
        }
    __syncthreads();

    // split-phase grid barrier: arrive once the CTA's partials are in global memory, do local work,
    // then wait (every CTA arrives at every barrier before it waits at it)
    // (the signal comes from kIdleThread, so its wait for the CTA's writes to be visible stalls no
    // warp that has work)
    auto arrive = [&]() {
        __syncthreads();
        if (threadIdx.x == kIdleThread) red_release_add_u32(&p.bar->count, 1u);
    };
    // a counter kIdleThread already saw complete spares the poll's round trip
    auto wait = [&]() -> bool {
        if (threadIdx.x == 0) {
            const unsigned int c = s_pre;
            s_ok = c >= (unsigned int)(epoch + 1) * G ? (c & kBarAbortBit) == 0 : grid_wait(p.bar, G, p.spin_limit, epoch);
            s_pre = 0u;
        }
        ++epoch;
        __syncthreads();
        return s_ok != 0;
    };
    // the polynomial's hooks: signal barrier A once the pass's partials are ordered before it, look
    // at the counter while the last product's rows are updated
    auto poly_hook = [&](int ev) {
        if (threadIdx.x != kIdleThread) return;
        if (ev == 0) red_release_add_u32(&p.bar->count, 1u);
        else s_pre = ld_acquire_u32(&p.bar->count);
    };
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
    auto cta_partials = [&](double a0, double a1, double a2, double a3, int i0, int i1) {
        a0 = bwarp_sum(a0); a1 = bwarp_sum(a1); a2 = bwarp_sum(a2); a3 = bwarp_sum(a3);
        if (lane == 0) { s_red[4 * warp] = a0; s_red[4 * warp + 1] = a1; s_red[4 * warp + 2] = a2; s_red[4 * warp + 3] = a3; }
        __syncthreads();
        if ((int)threadIdx.x >= i0 && (int)threadIdx.x < i1) {
            double t = 0.0;
            for (int w = 0; w < kWarps; ++w) t += s_red[4 * w + threadIdx.x];
            p.pdot[4 * cta + threadIdx.x] = t;
        }
    };
    // the dots of all CTAs, summed in CTA order (same bits everywhere): the last warp sums slots
    // 0-1, the one before it slots 2-3; every load is issued before the first add waits
    auto sum_dots = [&]() {
        if (warp < kWarps - 2) return;
        const int half = warp == kWarps - 1 ? 0 : 1;
        const double2* pd = reinterpret_cast<const double2*>(p.pdot) + half;
        constexpr int kB = 5;
        double2 v[kB];
#pragma unroll
        for (int i = 0; i < kB; ++i) {
            const unsigned c = lane + 32 * i;
            v[i] = c < G ? __ldcg(pd + 2 * c) : make_double2(0.0, 0.0);
        }
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int i = 0; i < kB; ++i) { a0 += v[i].x; a1 += v[i].y; }
        for (unsigned c = lane + 32 * kB; c < G; c += 32) {
            const double2 w = __ldcg(pd + 2 * c);
            a0 += w.x; a1 += w.y;
        }
        a0 = bwarp_sum(a0);
        a1 = bwarp_sum(a1);
        if (lane == 0) { s_dot[2 * half] = a0; s_dot[2 * half + 1] = a1; }
    };
    // out[j] = sum of column j's packed contributor partials, for every j < k: a warp per column,
    // its lanes over the partials (each lane adds its partials in order, then a fixed butterfly),
    // the loads of seven columns' first 64 slots in flight per warp before any add waits.  With
    // `dots` the last two warps sum the dots instead.
    auto sum_cols = [&](const double* part, double* out, bool dots) {
        const int nw = dots ? kWarps - 2 : kWarps;
        if (dots) sum_dots();
        if (warp >= nw || ncols == 0) return;  // a CTA without columns reads no sum (K s, C vt are per column)
        constexpr int kC = 7;
        for (int j0 = 0; j0 < k; j0 += kC * nw) {
            double a[kC], b2[kC];
#pragma unroll
            for (int i = 0; i < kC; ++i) {
                const int j = j0 + warp + nw * i;
                a[i] = 0.0;
                b2[i] = 0.0;
                if (j < k) {
                    const int q = s_srng[2 * j] + lane, q1 = s_srng[2 * j + 1];
                    if (q < q1) a[i] = __ldcg(part + q);
                    if (q + 32 < q1) b2[i] = __ldcg(part + q + 32);
                }
            }
#pragma unroll
            for (int i = 0; i < kC; ++i) {
                const int j = j0 + warp + nw * i;
                a[i] += b2[i];
                if (j < k)
                    for (int q = s_srng[2 * j] + 64 + lane; q < s_srng[2 * j + 1]; q += 32)
                        a[i] += __ldcg(part + q);
            }
#pragma unroll
            for (int i = 0; i < kC; ++i) {
                const double t = bwarp_sum(a[i]);
                const int j = j0 + warp + nw * i;
                if (lane == 0 && j < k) out[j] = t;
            }
        }
    };
    // out[q] = (M vin)_{s_cols[q]} for the CTA's columns, M = K or C (rows in registers when kreg)
    auto rows_times = [&](const double (&rg)[kRegCols][kRegK], const double* Mg, const double* vin, double* out) {
        if (kreg) {
#pragma unroll
            for (int c = 0; c < kRegCols; ++c) {
                const int q = warp + kWarps * c;
                if (q < ncols) {  // warp-uniform
                    double a = 0.0;
#pragma unroll
                    for (int i = 0; i < kRegK; ++i) {
                        const int l = lane + 32 * i;
                        a += rg[c][i] * (l < k ? vin[l] : 0.0);
                    }
                    a = bwarp_sum(a);
                    if (lane == 0) out[q] = a;
                }
            }
        } else {
            for (int q = warp; q < ncols; q += kWarps) {
                const int j = s_cols[q];
                double a = 0.0;
                for (int l = lane; l < k; l += 32) a += Mg[(size_t)j * p.kmax + l] * vin[l];
                a = bwarp_sum(a);
                if (lane == 0) out[q] = a;
            }
        }
    };
    // the CTA's Y columns at its own dofs: shared memory (FP32) when staged
    const float* Yc = reinterpret_cast<const float*>(sm + p.cta_yc[2 * cta]);
    auto yval = [&](int q, int e) -> double {
        if (q < nyc) return (double)Yc[(size_t)q * R3 + e];
        return (double)__ldg(p.Y + (size_t)s_cols[q] * 4 * p.n + 4 * (size_t)(sl.rb + e / 3) + e % 3);
    };
    // partials of Y^T v over the own dofs -> part[slot][j] for the CTA's columns
    auto y_partials = [&](const double* v, double* part) {
        for (int q = warp; q < ncols; q += kWarps) {
            double a = 0.0;
            for (int e = lane; e < R3; e += 32) a += yval(q, e) * v[e];
            a = bwarp_sum(a);
            if (lane == 0) part[s_slot[q]] = a;
        }
    };
    // the CTA's coupled rows of V, compact ([list position][own coupled dof], written by the Y kernel)
    const double* Vc = p.Vc + (size_t)p.kmax * sl.ab;
    // phase 2 copies the first nvs values of these rows into the segment scratch (free from the
    // polynomial's end to the local operator blocks), so V^T m reads shared memory
    const int nvs = min(ncols * sl.na, 3 * kSliceRows * (kWarps + p.NS));
    auto stage_v = [&]() {
        for (int i = threadIdx.x; i < nvs; i += blockDim.x) cp_async8(scr + i, Vc + i);
    };
    // partials of V^T v over the own coupled dofs (staged values first)
    auto v_partials = [&](const double* v, double* part) {
        if (sl.na == 0) return;
        for (int q = warp; q < ncols; q += kWarps) {
            const int f0 = q * sl.na;
            // the column's first 256 coupled dofs: every load in flight before the first add
            constexpr int kPre = 8;
            double vv[kPre];
#pragma unroll
            for (int u = 0; u < kPre; ++u) {
                const int il = lane + 32 * u, f = f0 + il;
                vv[u] = il < sl.na ? (f < nvs ? scr[f] : __ldg(Vc + f)) : 0.0;
            }
            double a = 0.0;
#pragma unroll
            for (int u = 0; u < kPre; ++u) {
                const int il = lane + 32 * u;
                if (il < sl.na) a += vv[u] * v[s_act[il]];
            }
            for (int il = lane + 32 * kPre; il < sl.na; il += 32) {
                const int f = f0 + il;
                a += (f < nvs ? scr[f] : __ldg(Vc + f)) * v[s_act[il]];
            }
            a = bwarp_sum(a);
            if (lane == 0) part[s_slot[q]] = a;
        }
    };
    // out[own coupled dof] -= (V s_t) (s_t = C vt on the CTA's columns)
    auto lowrank_sub = [&](double* out) {
        for (int il = threadIdx.x; il < sl.na; il += blockDim.x) {
            double a = 0.0, b = 0.0;
            int q = 0;
            for (; q + 8 <= ncols; q += 8) {
                double vv[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) vv[u] = __ldg(Vc + (size_t)(q + u) * sl.na + il);
#pragma unroll
                for (int u = 0; u < 8; u += 2) { a += vv[u] * s_t[q + u]; b += vv[u + 1] * s_t[q + u + 1]; }
            }
            for (; q < ncols; ++q) a += __ldg(Vc + (size_t)q * sl.na + il) * s_t[q];
            out[s_act[il]] -= a + b;
        }
    };
    // stage the halo of a published vector (the window's nodes outside the part; the remote pass
    // reads no others) and sum the V^T v partials into s_vt: the window loads (two per thread in
    // registers) are issued first, so they are in flight while the column sums wait on theirs
    auto stage_and_sum = [&](const double* pub, const double* part) {
        double wv[2][3];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int e = threadIdx.x + kThreads * i;
            wv[i][0] = wv[i][1] = wv[i][2] = 0.0;
            const int node = e < sl.nwin ? sl.wn[e] : sl.rb;
            if (node < sl.rb || node >= sl.re) {
                const double2 lo = __ldcg(reinterpret_cast<const double2*>(pub) + 2 * (size_t)node);
                wv[i][0] = lo.x; wv[i][1] = lo.y; wv[i][2] = __ldcg(pub + 4 * (size_t)node + 2);
            }
        }
        sum_cols(part, s_vt, false);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int e = threadIdx.x + kThreads * i;
            if (e < sl.nwin) { win[3 * e] = wv[i][0]; win[3 * e + 1] = wv[i][1]; win[3 * e + 2] = wv[i][2]; }
        }
        for (int e = threadIdx.x + 2 * kThreads; e < sl.nwin; e += blockDim.x) {
            const int node = sl.wn[e];
            if (node >= sl.rb && node < sl.re) continue;
            const double2 lo = __ldcg(reinterpret_cast<const double2*>(pub) + 2 * (size_t)node);
            win[3 * e] = lo.x; win[3 * e + 1] = lo.y; win[3 * e + 2] = __ldcg(pub + 4 * (size_t)node + 2);
        }
    };
    // n = S v over the own rows: D v (the local blocks, then the halo's) - V (C vt), vt = V^T v
    // summed from `part`
    auto schur_apply = [&](const double* pub, const double* vown, const double* part) {
        part_op_local<MT>(sl, s_plan_loc, scr, gv, vown, Nn);
        stage_and_sum(pub, part);
        __syncthreads();
        part_op_remote<MT>(sl, s_plan_rem, scr, gv, win, Nn);
        rows_times(cr, p.C, s_vt, s_t);
        __syncthreads();
        lowrank_sub(Nn);
        __syncthreads();
    };

    // ---- prologue: x = 0, r = rhs, the first pass preconditions r ----
    double xr[kDofs], rr_[kDofs], ur[kDofs];
#pragma unroll
    for (int i = 0; i < kDofs; ++i) {
        const int e = threadIdx.x + kThreads * i;
        xr[i] = ur[i] = rr_[i] = 0.0;
        if (e < R3) {
            rr_[i] = p.rhs[4 * (size_t)(sl.rb + e / 3) + e % 3];
            Wb[e] = rr_[i];
            Zv[e] = Qv[e] = Sv[e] = Pv[e] = 0.0;
        }
    }
    __syncthreads();

    int pass = kPassStart, it = 0, status = -1, restarts = 0, npass = 0;
    // phase clocks (trace mode): 0 pass top, 1 Y^T v and dot partials written (arrive A), 2 polynomial
    // done, 3 after wait A, 4 sums read, 5 K s done, 6 m formed, 7 V^T m partials / decisions (arrive
    // B), 8 local operator blocks and early recurrences done, 9 after wait B, 10 halo staged and V^T m
    // summed, 11 halo blocks and C vt done, 12 low-rank done, 13 updates done
    auto mark = [&](int ev) {
        if (p.trace && threadIdx.x == 0 && npass < p.trace_iters)
            p.trace[((size_t)cta * p.trace_iters + npass) * 16 + ev] = (unsigned long long)clock64();
    };
    double normb = -1.0, rel = 1.0, alpha = 0.0, beta = 0.0, alpha_prev = 0.0, gamma_prev = 0.0;
    bool fresh = true;  // next normal pass is the first after a (re)start: beta = 0
    for (;;) {
        // ---------------- phase 1: partials, arrive A, the polynomial, wait A ----------------
        mark(0);
        y_partials(Wb, p.pY);
        {
            double g = 0, d = 0, rr = 0;
#pragma unroll
            for (int i = 0; i < kDofs; ++i) {
                const int e = threadIdx.x + kThreads * i;
                if (e < R3) {
                    rr += rr_[i] * rr_[i];
                    if (pass == kPassNormal) { g += rr_[i] * ur[i]; d += Wb[e] * ur[i]; }
                }
            }
            cta_partials(g, d, rr, 0.0, 0, 3);
        }
        mark(1);
        part_poly_bal<MT>(p, sl, s_plan_loc, scr, Wb, Pz, Pt, Pu, poly_hook);
        mark(2);
        if (!wait()) return;
        mark(3);
        // ---------------- phase 2 ----------------
        stage_v();
        sum_cols(p.pY, s_sv, true);
        __syncthreads();
        mark(4);
        rows_times(kr, p.K, s_sv, s_c);
        __syncthreads();
        mark(5);
#pragma unroll
        for (int i = 0; i < kDofs; ++i) {
            const int e = threadIdx.x + kThreads * i;
            if (e < R3) {
                const int lr = e / 3, d = e - 3 * lr;
                double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;  // four chains over the columns
                int q = 0;
                if (ncols <= nyc) {  // every column staged: plain shared-memory loads
                    const float* yc = Yc + e;
                    for (; q + 4 <= ncols; q += 4) {
                        m0 += (double)yc[(size_t)q * R3] * s_c[q];
                        m1 += (double)yc[(size_t)(q + 1) * R3] * s_c[q + 1];
                        m2 += (double)yc[(size_t)(q + 2) * R3] * s_c[q + 2];
                        m3 += (double)yc[(size_t)(q + 3) * R3] * s_c[q + 3];
                    }
                    for (; q < ncols; ++q) m0 += (double)yc[(size_t)q * R3] * s_c[q];
                } else {
                    for (; q + 4 <= ncols; q += 4) {
                        m0 += yval(q, e) * s_c[q];
                        m1 += yval(q + 1, e) * s_c[q + 1];
                        m2 += yval(q + 2, e) * s_c[q + 2];
                        m3 += yval(q + 3, e) * s_c[q + 3];
                    }
                    for (; q < ncols; ++q) m0 += yval(q, e) * s_c[q];
                }
                const double m = Pz[e] + ((m0 + m1) + (m2 + m3));
                Mm[e] = m;
                p.mpub[4 * (size_t)(sl.rb + lr) + d] = m;
            }
        }
        cp_async_wait_all();  // the staged V rows
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
        // ---------------- arrive B, local work, wait B, phase 3 ----------------
        arrive();
        if (!check) {
            // n's blocks inside the part, and the recurrences that do not need n:
            // q = m + b q, s = w + b s, p = u + b p, x += a p, r -= a s, u -= a q (a start takes u = m)
            part_op_local<MT>(sl, s_plan_op, scr, gv, Mm, Nn);
#pragma unroll
            for (int i = 0; i < kDofs; ++i) {
                const int e = threadIdx.x + kThreads * i;
                if (e < R3) {
                    if (pass == kPassStart) {
                        ur[i] = Mm[e];
                    } else {
                        const double q = Mm[e] + beta * Qv[e], sv = Wb[e] + beta * Sv[e], pv = ur[i] + beta * Pv[e];
                        Qv[e] = q; Sv[e] = sv; Pv[e] = pv;
                        xr[i] += alpha * pv;
                        rr_[i] -= alpha * sv;
                        ur[i] -= alpha * q;
                    }
                }
            }
        }
        mark(8);
        if (!wait()) return;
        mark(9);
        if (!check) {
            stage_and_sum(p.mpub, p.pV);
            __syncthreads();
            mark(10);
            part_op_remote<MT>(sl, s_plan_rem, scr, gv, win, Nn);
            rows_times(cr, p.C, s_vt, s_t);
            __syncthreads();
            mark(11);
            lowrank_sub(Nn);
            __syncthreads();
            mark(12);
            // the rest: z = n + b z, w -= a z (a start takes w = n)
#pragma unroll
            for (int i = 0; i < kDofs; ++i) {
                const int e = threadIdx.x + kThreads * i;
                if (e < R3) {
                    if (pass == kPassStart) {
                        Wb[e] = Nn[e];
                    } else {
                        const double z = Nn[e] + beta * Zv[e];
                        Zv[e] = z;
                        Wb[e] -= alpha * z;
                    }
                }
            }
            if (pass == kPassStart) {
                pass = kPassNormal;
                fresh = true;
            } else {
                ++it;
                fresh = false;
            }
            __syncthreads();
            mark(13);
            ++npass;
            continue;
        }
        // ---------------- true residual: r = rhs - (D x - V C V^T x) ----------------
#pragma unroll
        for (int i = 0; i < kDofs; ++i) {
            const int e = threadIdx.x + kThreads * i;
            if (e < R3) {
                Mm[e] = xr[i];
                p.xpub[4 * (size_t)(sl.rb + e / 3) + e % 3] = xr[i];
            }
        }
        __syncthreads();
        v_partials(Mm, p.pX);
        if (!barrier()) return;
        schur_apply(p.xpub, Mm, p.pX);
        {
            double rr = 0.0;
#pragma unroll
            for (int i = 0; i < kDofs; ++i) {
                const int e = threadIdx.x + kThreads * i;
                if (e < R3) {
                    rr_[i] = p.rhs[4 * (size_t)(sl.rb + e / 3) + e % 3] - Nn[e];
                    rr += rr_[i] * rr_[i];
                }
            }
            cta_partials(0.0, 0.0, 0.0, rr, 3, 4);
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
#pragma unroll
        for (int i = 0; i < kDofs; ++i) {
            const int e = threadIdx.x + kThreads * i;
            if (e < R3) Wb[e] = rr_[i];
        }
        __syncthreads();
    }
    // ---- x out (own rows) and the scalars ----
#pragma unroll
    for (int i = 0; i < kDofs; ++i) {
        const int e = threadIdx.x + kThreads * i;
        if (e < R3) {
            const size_t o = 4 * (size_t)(sl.rb + e / 3) + e % 3;
            p.x[o] = xr[i];
            if (e % 3 == 2) p.x[o + 1] = 0.0;  // the node's pad
        }
    }
    if (cta == 0 && threadIdx.x == 0) {
        p.out[0] = it; p.out[1] = rel; p.out[2] = status; p.out[3] = normb; p.out[4] = restarts;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_block_fill(int precision, const BlockPlan& p, cudaStream_t st) {
    const long long nslot = p.nchunk * 32;
    if (nslot <= 0) return;
    const int grid = (int)std::min<long long>((nslot + 255) / 256, 148LL * 8);
    count_launch();
    if (precision == 0) block_fill_kernel<double><<<grid, 256, 0, st>>>(p);
    else block_fill_kernel<float><<<grid, 256, 0, st>>>(p);
}

void launch_block_columns(const BlockPlan& p, cudaStream_t st) {
    count_launch();
    block_columns_kernel<<<1, 1024, 0, st>>>(p);
}

template <class MT>
static cudaError_t launch_y_t(const BlockPlan& p, cudaStream_t st) {
    auto fn = block_y_kernel<MT>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_y);
    if (e != cudaSuccess) return e;
    const size_t gsm = p.gpart_staged ? gpart_smem_bytes(p.kmax, p.NA, p.NCOL) : gpart_stage_offset(p.kmax);
    e = cudaFuncSetAttribute(block_gpart_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm);
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(p.Yact, 0, sizeof(double) * (size_t)p.a * p.kmax, st);
    const int batches = std::max(1, (p.NCOL + kYBatch - 1) / kYBatch);
    BlockPlan py = p;  // the Y kernel's value chunks follow its own vector region
    py.off_val = p.off_val_y;
    count_launch();
    fn<<<dim3(p.G_ctas, batches), kThreads, p.smem_y, st>>>(py);
    count_launch();
    block_gpart_kernel<<<p.G_ctas, kThreads, gsm, st>>>(p);
    return cudaPeekAtLastError();
}

cudaError_t launch_block_y(int precision, const BlockPlan& p, cudaStream_t st) {
    return precision == 0 ? launch_y_t<double>(p, st) : launch_y_t<float>(p, st);
}

void launch_block_g(const BlockPlan& p, int nact_cta, cudaStream_t st) {
    const int kk = p.kmax * p.kmax;
    count_launch();
    block_g_reduce_kernel<<<(kk + 255) / 256, 256, 0, st>>>(p.pG, nact_cta, kk, p.G);
}

void launch_block_k(const BlockPlan& p, cudaStream_t st) {
    const int kk = p.kmax * p.kmax;
    const int* dk = p.rank;
    // Ka = G Lc, Kb = Lc^T Ka
    GemmArgs g1{p.G, p.Lc, p.Ka, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 0, 0, 1.0, 0.0};
    launch_gemm(g1, p.kmax, p.kmax, st);
    GemmArgs g2{p.Lc, p.Ka, p.Kb, p.kmax, p.kmax, p.kmax, dk, dk, dk, p.kmax, p.kmax, p.kmax, 1, 0, 1.0, 0.0};
    launch_gemm(g2, p.kmax, p.kmax, st);
    count_launch();
    block_kinv_kernel<<<(kk + 255) / 256, 256, 0, st>>>(p.Kb, p.dpiv, dk, p.kmax, p.Ka);
    // K~ = (K^-1)^-1 into Kb (Cholesky: flags a matrix that is not SPD)
    cudaMemsetAsync(p.bad, 0, sizeof(int), st);
    if (!launch_chol_inverse(p.Ka, p.kmax, p.Kb, p.bad, st, dk)) {
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

// the kernels' own static shared memory (the plan copy, reductions) is kept out of the budget
int block_max_smem() { return 227 * 1024 - 8 * 1024; }

// shared-memory layouts for the maxima in p (R, NS, NCH, W, NA, NCOL, kmax): a common prefix
// (slices, local slot counts, window positions, Dd^-1, window, coupled dofs and their diagonal
// blocks, column lists and slot ranges, k-vectors, reduction scratch), then for the PCG its eight
// FP64 vectors (3 per row), the segment scratch and the CTA's value chunks, after which each CTA
// stages its Y columns (FP32) at its own offset (cta_yc, set by the host: a small part leaves room
// for more columns); for the Y kernel its batch region, then the value chunks.  Returns the PCG's
// bytes without Y columns and sets smem_y.
size_t block_smem_bytes(int precision, BlockPlan& p, bool stage_vals) {
    const size_t mt = precision == 0 ? 8 : 4, dt = mt;
    auto al = [](size_t b) { return (b + 15) / 16 * 16; };
    size_t off = 0;
    p.off_meta = (int)off; off += al(sizeof(int4) * p.NS);
    p.off_nloc = (int)off; off += al(sizeof(unsigned short) * p.R);
    p.off_lc = (int)off; off += al(sizeof(unsigned short) * 32 * (size_t)p.NCH);
    p.off_dinv = (int)off; off += al(dt * 9 * p.R);
    p.off_wn = (int)off; off += al(sizeof(int) * p.W);
    p.off_win = (int)off; off += al(sizeof(double) * 3 * p.W);
    p.off_act = (int)off; off += al(sizeof(int) * p.NA);
    p.off_aflag = (int)off; off += al(sizeof(int) * p.R);
    p.off_dact = (int)off; off += al(sizeof(double) * 3 * p.NA);
    p.off_cols = (int)off; off += al(sizeof(int) * 2 * p.kmax);
    p.off_srng = (int)off; off += al(sizeof(int) * 2 * p.kmax);
    p.off_kv = (int)off; off += al(sizeof(double) * 4 * p.kmax);
    p.off_red = (int)off; off += al(sizeof(double) * 4 * kWarps);
    p.off_vec = (int)off;
    p.stage_vals = stage_vals ? 1 : 0;
    const size_t vals = stage_vals ? al(mt * kChunkVals * (size_t)p.NCH) : 0;
    p.off_val_y = (int)(off + al(sizeof(double) * y_region_doubles(p.R)));
    p.smem_y = p.off_val_y + vals;
    off += al(sizeof(double) * 8 * 3 * (size_t)p.R);
    p.off_scr = (int)off;
    off += al(sizeof(double) * 3 * kSliceRows * (size_t)(kWarps + p.NS));
    p.off_val = (int)off;
    off += vals;
    p.smem = off;
    p.gpart_staged = gpart_smem_bytes(p.kmax, p.NA, p.NCOL) <= (size_t)block_max_smem() ? 1 : 0;
    return off;
}

}  // namespace hsc
