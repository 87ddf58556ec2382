// Block-local Woodbury preconditioner and pipelined Schur PCG (hsc_block.cu).
//
// The Schur operator is the reference's, S = D - V C V^T (linear_hsc.cu:306-329,
// with C = U^T P U).  The preconditioner is this build's own:
//
//   M^-1 r = L r + Y K Y^T r,   Y = L V,   K = (C^-1 - V^T Y)^-1,
//
// where L is a polynomial in w Dd^-1 D_loc, D_loc keeping only the blocks
// whose two nodes lie in the same part (one part = one PCG CTA's rows), so a
// term needs no grid barrier: each CTA applies it to its own rows from shared
// memory.  By the Woodbury identity M = L^-1 - V C V^T: with L = D^-1 this is
// S^-1 exactly, so the coupling's soft modes, which no polynomial in D reaches,
// cost the PCG nothing and it iterates only against the polynomial's error.
//
// V's columns come from the ACA of the coupling E.  E is block-structured by
// coupling component (bodies linked through the FEM nodes they share): a
// full-pivot ACA step never mixes components, so every column of U and V lives
// on one component.  A part touches few components (a rim, the ground), so
// Y = L V restricted to a part has few nonzero columns, and the reductions of
// Y^T v and V^T v over the CTAs only sum the CTAs that hold a component's
// nodes (its contributor slots).
//
// K is formed from the LDL^T factors of C (C = L_c diag(d) L_c^T) as
// K = L_c (diag(1/d) - L_c^T G L_c)^-1 L_c^T, G = V^T Y, which avoids
// inverting C itself; when diag(1/d) - L_c^T G L_c is not SPD the correction is
// dropped (K = 0) and M^-1 = L.
//
// PCG: Ghysels & Vanroose's pipelined form, two grid barriers per iteration
// (one for the Y^T w reduction of m = M w, one for the halo of m and the
// V^T m reduction of n = S m), the dot products riding on the first.
#pragma once
#include "hsc_internal.cuh"

namespace hsc {

struct BlockPlan {
    // system (internal FEM node numbering)
    int n, nnz, a, kmax;
    const int* rank;             // device rank k
    const void* vals;            // BSR operator planes 9 x nnz (MT); mixed modes: coupled diagonal blocks zeroed
    const void* dinv;            // Dd^-1 planes over nodes (DT)
    const double* dact;          // FP64 diagonal blocks of the coupled nodes, actp node order (mixed modes)
    const int* rowflag;          // node -> coupled-node index in actp order, or -1
    const int* actp;             // coupled dofs, internal numbers, sorted (a)
    const int* actperm;          // actp position -> row of V (the caller's active order)
    const double* V;             // a x kmax, column-major
    const double* C;             // kmax x kmax, row-major, C = U^T P U
    const double* Lc;            // kmax x kmax, row-major unit lower LDL^T factor of C
    const double* dpiv;          // LDL^T pivots
    const double* U;             // qm x kmax, column-major (component of each column)
    int qm;
    double* K;                   // kmax x kmax, row-major Woodbury core
    double* Ka;                  // kmax x kmax scratch
    double* Kb;                  // kmax x kmax scratch
    float* Y;                    // kmax columns of 4n node-padded rows (column-major)
    double* Yact;                // a x kmax, column-major, actp order: Y at the coupled dofs
    double* Vc;                  // per CTA at kmax * ab: its coupled rows of V, [column in its list][dof]
    double* pG;                  // per coupled CTA: kmax x kmax partial of V^T Y
    double* G;                   // kmax x kmax
    int* bad;                    // device flags: [0] K^-1 not SPD
    const double* ident;         // kmax x kmax identity (the Cholesky-solve path of large ranks)
    // partition (one CTA per part) and the CTAs' vector windows
    int G_ctas;
    const int* cta_row;          // [rb, re) per CTA
    const int* cta_act;          // [ab, ae) per CTA in actp
    const int* cta_aidx;         // index among the CTAs with coupled dofs, or -1
    const int* win_off;
    const int* win_nodes;
    const int* win_own;
    // sliced ELL of the CTAs' rows: slices of 16 rows, two slots of each row per 32-lane chunk
    // (lane 2 r + h holds slot 2 c + h of row r in chunk c); a row's slots are its diagonal block,
    // then the blocks whose column is a row of the same part, then the rest, then zero padding
    const int4* sell_slice;      // per slice: first chunk, chunks, chunks holding local slots, first chunk holding a remote one
    const int* cta_slice;        // G + 1: each CTA's slices
    const int* cta_chunk;        // G + 1: each CTA's chunks
    const unsigned short* sell_nloc;  // per row: its diagonal block + local blocks (leading slots)
    const unsigned short* sell_lc;    // per slot: window position of the block's column
    const int* sell_src;         // per slot: BSR entry, or -1 for padding
    void* sell_vals;             // per chunk kChunkVals MT: planes 0-3 as [lane][4], 4-7 as [lane][4], 8 as [lane]
    long long nchunk;            // chunks over all CTAs
    // coupling components
    int ncomp;
    const int* comp_of_body;     // body -> component
    const int* cta_comp_ptr;     // G + 1
    const int* cta_comp;         // the components with a coupled node in each CTA's part
    const int* cta_comp_slot;    // that CTA's slot in the component's contributor list
    const int* comp_slot_ptr;    // ncomp + 1 (slots = contributor CTAs of each component)
    int nslot;
    int* comp_of_col;            // kmax (set after the ACA), -1 for unused columns
    int* comp_col_ptr;           // ncomp + 1
    int* comp_cols;              // kmax
    int* col_off;                // kmax + 1: column j's contributor partials are pY[col_off[j] .. col_off[j + 1])
    // vectors (node-padded FP64)
    double* x;                   // solution (written)
    const double* rhs;           // Schur right-hand side
    double* mpub;                // m published for the neighbours' windows
    double* xpub;                // x published for the true-residual check
    // partials, packed by column (col_off), each column's in its component's slot order
    double* pY;                  // Y^T v
    double* pV;                  // V^T m
    double* pX;                  // V^T x (true-residual check)
    double* pdot;                // G x 4
    // polynomial
    int nterms;
    double omega;
    double w[16];
    const double* wdev;          // device weights (learned), or null
    // control
    double tol;
    int max_iter;
    int rr_every;
    long long spin_limit;
    GridBar* bar;
    double* out;                 // iterations, relative residual, status, |rhs|, restarts
    double* cg_coef;             // alpha_i, beta_{i+1} pairs (Lanczos of the preconditioned operator)
    int max_coef;
    unsigned long long* trace;   // optional: per CTA x trace_iters x 16 SM clocks at the phase boundaries
    int trace_iters;
    // shared-memory layout (bytes from the dynamic base, the same in every CTA but for the Y
    // columns, which follow the CTA's own value chunks)
    int R, NS, NCH, W, NA, NCOL; // maxima over CTAs: rows, slices, chunks, window nodes, coupled dofs, Y columns
    int stage_vals, NYC, gpart_staged;  // value chunks staged; the most Y columns a CTA stages
    int off_meta, off_nloc, off_lc, off_val, off_dinv, off_wn, off_win, off_act, off_aflag, off_dact;
    int off_cols, off_srng, off_kv, off_red, off_vec, off_scr;
    int off_val_y;               // the Y kernel's value chunks (after its larger vector region)
    const int* cta_yc;           // per CTA: byte offset of its staged Y columns, how many it stages
    size_t smem;                 // the PCG kernel
    size_t smem_y;               // the Y kernel
};

constexpr int kSliceRows = 16;
constexpr int kChunkVals = 9 * 32;
constexpr int kBlockMaxRows = 341;  // the PCG keeps a CTA's dofs in registers, two per thread

// sliced-ELL values from the BSR planes (every solve)
void launch_block_fill(int precision, const BlockPlan& p, cudaStream_t st);
// columns of every coupling component, from U's nonzero rows (after the ACA)
void launch_block_columns(const BlockPlan& p, cudaStream_t st);
// Y = L V over every part, Y at the coupled dofs, and the per-CTA partials of V^T Y
cudaError_t launch_block_y(int precision, const BlockPlan& p, cudaStream_t st);
// G = the sum of the coupled CTAs' partials of V^T Y (fixed order)
void launch_block_g(const BlockPlan& p, int nact_cta, cudaStream_t st);
// K^-1 = diag(1/d) - L_c^T G L_c, K = L_c K~ L_c^T (K = 0 if not SPD)
void launch_block_k(const BlockPlan& p, cudaStream_t st);
// the persistent pipelined PCG (cooperative launch, one CTA per part)
cudaError_t launch_block_pcg(int precision, const BlockPlan& p, cudaStream_t st);
// shared-memory layouts of the two block kernels for the maxima in p; returns the larger
size_t block_smem_bytes(int precision, BlockPlan& p, bool stage_vals);
int block_max_smem();

}  // namespace hsc
