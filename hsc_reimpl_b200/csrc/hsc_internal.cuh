// Internal declarations of the B200 HSC solver (device data layout, kernels,
// the bounded grid barrier).  Host orchestration lives in hsc_api.cu.
//
// Device layout of one system (all FP64 unless the precision mode says
// otherwise):
//   * FEM block D as a full (both-triangle) row-owner BSR over nodes:
//     rowptr[n+1], colidx[nnz], and the 3x3 values as 9 planes
//     vals[e*nnz + k] (e = 3*r + c, row-major inside the block) so that the
//     lanes of one row read consecutive k of a plane: coalesced.
//   * 3x3 diagonal-block inverses Dinv as 9 planes over nodes.
//   * FEM vectors padded to 4 entries per node (x, y, z, 0): one 32-byte
//     (FP64) or 16-byte (FP32) aligned load per node in the gathers.
//   * low-rank coupling: sorted active FEM dofs act[a], Vt = V L (a x kmax,
//     column-major) and the LDL^T pivots dpiv[kmax] of C = U^T P U, so that
//     V C V^T = Vt diag(dpiv) Vt^T.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace hsc {

constexpr int kThreads = 512;            // persistent-kernel CTA size (one CTA per SM)
constexpr int kWarps = kThreads / 32;
constexpr int kMaxRank = 256;

struct GridBar {
    unsigned int count;
    unsigned int gen;
    int abort;
    int where;                           // phase id of the wait that gave up
};

// ----------------------------------------------------------------------------
// memory-order helpers
// ----------------------------------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned int* p, unsigned int v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}
__device__ __forceinline__ void red_release_add_u32(unsigned int* p, unsigned int v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread-0 half of a grid barrier: release-arrive on the monotonic counter,
// then acquire-poll until barrier `epoch` is complete.  Bounded: returns
// false (and raises gb->abort) when the wait gives up or another CTA aborted.
// A CTA that gives up also sets the counter's top bit, so every waiter's poll
// sees the count reach its target and the abort in the same load: the barrier
// costs no extra round trip for the abort check.  (The counter is reset before
// each launch and stays below 2^31: epochs x CTAs per launch.)
constexpr unsigned int kBarAbortBit = 0x80000000u;
// The wait half alone serves a split-phase barrier: the CTA arrived earlier
// (red_release_add_u32 on gb->count after a CTA-wide barrier) and did local
// work in between.
__device__ __forceinline__ bool grid_wait(GridBar* gb, unsigned int nblocks, long long limit, int epoch) {
    const unsigned int target = (unsigned int)(epoch + 1) * nblocks;
    long long n = 0;
    unsigned int c;
    while ((c = ld_acquire_u32(&gb->count)) < target) {
        ++n;
        if (n > 256) __nanosleep(20);
        if (n > limit) {
            atomicExch(&gb->abort, 1);
            atomicExch(&gb->where, epoch);
            atomicOr(&gb->count, kBarAbortBit);
            return false;
        }
    }
    return (c & kBarAbortBit) == 0;
}

__device__ __forceinline__ bool grid_arrive_wait(GridBar* gb, unsigned int nblocks, long long limit, int epoch) {
    const unsigned int target = (unsigned int)(epoch + 1) * nblocks;
    red_release_add_u32(&gb->count, 1u);
    long long n = 0;
    unsigned int c;
    while ((c = ld_acquire_u32(&gb->count)) < target) {
        ++n;
        if (n > 256) __nanosleep(20);
        if (n > limit) {
            atomicExch(&gb->abort, 1);
            atomicExch(&gb->where, epoch);
            atomicOr(&gb->count, kBarAbortBit);
            return false;
        }
    }
    return (c & kBarAbortBit) == 0;
}

// Grid-wide barrier for a cooperative launch.  The arrival counter only
// grows: barrier number `epoch` (0, 1, 2, ... per launch) completes when it
// reaches (epoch + 1) * nblocks, so no reset round trip is needed.  Every wait
// is bounded by `limit` polls; a wait that gives up raises gb->abort, after
// which every CTA leaves at its next barrier.  Returns false when the grid
// must exit.
__device__ __forceinline__ bool grid_sync(GridBar* gb, unsigned int nblocks, long long limit, int epoch) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int target = (unsigned int)(epoch + 1) * nblocks;
        __threadfence();
        atomicAdd(&gb->count, 1u);
        long long n = 0;
        while (ld_acquire_u32(&gb->count) < target) {
            ++n;
            if (n > 64) __nanosleep(32);
            if ((n & 127) == 0 && ld_volatile_i32(&gb->abort)) { ok = 0; break; }
            if (n > limit) {
                atomicExch(&gb->abort, 1);
                atomicExch(&gb->where, epoch);
                ok = 0;
                break;
            }
        }
        if (ld_volatile_i32(&gb->abort)) ok = 0;
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ----------------------------------------------------------------------------
// value types
// ----------------------------------------------------------------------------
template <class T> struct Num;
template <> struct Num<double> {
    __device__ __forceinline__ static double get(double v) { return v; }
    __device__ __forceinline__ static double put(double v) { return v; }
};
template <> struct Num<float> {
    __device__ __forceinline__ static float get(float v) { return v; }
    __device__ __forceinline__ static float put(double v) { return (float)v; }
};
template <> struct Num<__nv_bfloat16> {
    __device__ __forceinline__ static float get(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ __forceinline__ static __nv_bfloat16 put(double v) { return __float2bfloat16_rn((float)v); }
};

// node-padded vector element access: 4 entries per node
template <class VT> struct Vec4;
template <> struct Vec4<double> {
    __device__ __forceinline__ static void load(const double* v, int node, double& a, double& b, double& c) {
        const double2* q = reinterpret_cast<const double2*>(v + 4 * (size_t)node);
        double2 u = q[0];
        double2 w = q[1];
        a = u.x; b = u.y; c = w.x;
    }
    __device__ __forceinline__ static void store(double* v, int node, double a, double b, double c) {
        double2* q = reinterpret_cast<double2*>(v + 4 * (size_t)node);
        q[0] = make_double2(a, b);
        q[1] = make_double2(c, 0.0);
    }
};
template <> struct Vec4<float> {
    __device__ __forceinline__ static void load(const float* v, int node, float& a, float& b, float& c) {
        float4 u = reinterpret_cast<const float4*>(v)[node];
        a = u.x; b = u.y; c = u.z;
    }
    __device__ __forceinline__ static void store(float* v, int node, float a, float b, float c) {
        reinterpret_cast<float4*>(v)[node] = make_float4(a, b, c, 0.f);
    }
};

// ----------------------------------------------------------------------------
// per-system device descriptor used by the persistent PCG kernel
// ----------------------------------------------------------------------------
struct SysDesc {
    int n;                 // FEM nodes (block rows of D)
    int nnz;               // full BSR entries
    int a;                 // active FEM dofs (3 per active node)
    int kmax;              // allocated rank columns
    int cta_begin, cta_end;
    const int* rowflag;    // per node: active-node index, or -1
    const int* rowptr;
    const int* colidx;
    const int* rowid;      // block row of every BSR entry
    const void* vals;      // operator planes (mixed modes: active diagonal blocks zeroed)
    const void* vals_pc;   // preconditioner planes (BF16 mode: bf16 copy; else == vals)
    const double* vals64;  // FP64 planes (true-residual replacement)
    const double* dact;    // FP64 active diagonal blocks (mixed modes), row-major 9 per active node
    const void* dinv;      // Dd^-1 planes over nodes (omega NOT folded in)
    const int* act;        // active FEM dofs (a), sorted
    const double* vt64;    // Vt = V L (a x kmax, column-major), FP64
    const double* dpiv;    // LDL^T pivots (kmax)
    const int* rank;       // device scalar
    double* x;             // FP64 node-padded
    double* r;             // FP64 node-padded
    double* r2;            // second residual buffer (fused update: neighbours read the old r)
    const double* rhs;     // FP64 node-padded
    void* z;               // VT node-padded
    void* p[2];            // VT node-padded ping-pong
    void* y;               // VT node-padded
    void* t[2];            // VT node-padded ping-pong polynomial terms
    double* pact;          // FP64 direction at the active dofs (a)
    double* yact;          // FP64 S p at the active dofs (a)
    double* zpart;         // kmax x ncta: per-CTA partials of Vt^T z (own active dofs)
    double* tpart;         // 2 x kmax x nact_cta: partials of Vt^T t_k of the CTAs with coupled dofs
                           // (Schur-basis terms), by term parity
    int nact_cta;          // CTAs of this system that own coupled dofs
    const unsigned short* lcol;  // resident mode: per BSR entry, window position of its column
    const double* wdev;    // device polynomial weights of this system (learned), or null: PcgParams::w
    double* tt;            // kmax: Vt^T p (recurrence Vt^T z + beta Vt^T p_prev)
    double* ttx;           // kmax: Vt^T x (true-residual slot)
    double* out;           // per-system results [0]=iters [1]=rel [2]=status [3]=normb [4]=replacements
    double* cg_coef;       // 2*max_coef: alpha_k, beta_k for the Lanczos estimate
    int max_coef;
};

constexpr int kTraceEvents = 16;  // clock slots per CTA and iteration in trace mode
constexpr int kMaxCoef = 256;  // CG coefficients kept per solve for the Lanczos estimates

struct PcgParams {
    const SysDesc* sys;
    int nsys;
    const int* cta_sys;        // per CTA: its system
    const int* cta_row;        // per CTA: [row_begin, row_end) pairs
    const int* cta_act;        // per CTA: [act_begin, act_end) pairs in the system's act list
    const int* cta_aidx;       // per CTA: its index among the system's CTAs with coupled dofs, or -1
    double* part_rr;           // per CTA: r.r after the update phase
    double* part_rz;           // per CTA: r.z after the last preconditioner phase
    double* part_pap;          // per CTA: p.S p of phase A
    GridBar* bar;
    int* remaining;            // systems still iterating
    double omega;
    int nterms;                // polynomial terms (Neumann order or poly degree)
    double w[16];              // polynomial weights
    int schur_basis;           // terms t_k = (I - w Dd^-1 S)^k t_0 on the Schur operator (else on D)
    double tol;
    int max_iter;
    int rr_every;              // residual replacement interval (0 = only at convergence)
    long long spin_limit;
    const int* cta_warp;       // per CTA: kWarps + 1 row boundaries of the warp-owned row ranges
    // shared-memory layout (offsets in doubles from the dynamic base, the same in every CTA)
    int off_z, off_vt, off_y, off_blk;
    int stage_vt;              // the CTAs' Vt blocks are staged (else read from global)
    int stage_blk;             // the CTAs' column indices and row ids are staged
    int vt_smem;               // doubles reserved for the largest Vt block (pad(na) + na * rank)
    unsigned long long* trace; // optional: per CTA x trace_iters x 8 SM clocks
    int trace_iters;
    // resident mode: each CTA keeps its BSR slice (operator and preconditioner
    // planes), local indices and the window of vector nodes its blocks read in
    // shared memory; a phase stages the window once and runs the SpMV from there
    int resident;
    int stage_vals;            // resident mode: the value planes are copied too (else read from L2)
    const int* win_off;        // per CTA: G + 1 offsets into win_nodes
    const int* win_nodes;      // sorted global node ids of each CTA's window
    const int* win_own;        // per CTA: window position of its first row
    int off_wn, off_win, off_val, off_vpc, off_lidx;  // shared-memory offsets (doubles)
    int off_dinv, off_rf;      // the CTA's rows' Dd^-1 planes and row flags (resident mode)
    int off_own, off_act;      // own-row vectors (x, r, z, p, y, t) and coupled-dof values / list
    // fused update (resident mode, FEM-basis polynomial, normal slots): after the
    // alpha barrier every CTA forms t0 = w Dd^-1 (r - alpha y) over its window
    // itself, so the update and the first preconditioner phase share a barrier
    int fuse;
    const int* win_flag;       // per window entry: position in the CTA's coupled-window list, or -1
    const int* win_act_off;    // per CTA: G + 1 offsets into win_act
    const int* win_act;        // active-node index (rowflag) of each coupled window node
    int off_wflag, off_wact, off_wcorr, wact_max;
    int own_rows, own_act;     // rows and coupled dofs the own-row regions hold (the maxima over CTAs)
};

// launch counter of this library (hsc_setup.cu)
void count_launch();
long long launch_count();
// with HSC_SYNC_CHECK set: synchronise and report the first failing launch
void debug_sync(const char* what);

// kernel launchers (hsc_pcg.cu)
cudaError_t launch_pcg(int precision, int tpr, const PcgParams& prm, int grid, size_t smem, cudaStream_t st);
int pcg_blocks_per_sm(int precision, int tpr, size_t smem);
// dynamic shared memory of the PCG kernel for a Vt block of `vt_doubles`
size_t pcg_smem_bytes(int vt_doubles, int kmax_all);

}  // namespace hsc
