// Launchers of the numeric setup, dense-algebra and vector kernels (hsc_setup.cu).
#pragma once
#include <algorithm>

#include "hsc_internal.cuh"

namespace hsc {

struct AcaParams {
    double* R0;            // holds E on entry (row-major m x nc); overwritten
    double* R1;            // second buffer
    int m, nc, cap;
    double rtol;           // stop when |R|_F/|E|_F <= rtol (0: only the zero-pivot guard)
    double* U;             // m x cap, column-major
    double* V;             // nc x cap, column-major
    double* hist;          // cap + 1 residuals
    int* rank;
    double* err;
    double* psum;          // per-CTA partials
    double* pmax;
    long long* pidx;
    GridBar* bar;
    long long spin_limit;
    int strip;             // columns per CTA (set by launch_aca)
};

// one system of the cluster ACA (hsc_aca.cu)
struct AcaSys {
    const double* E;       // coupling, row-major m x nc (read only)
    int m, nc, cap;
    double rtol;
    double* U;             // m x cap, column-major
    double* V;             // nc x cap, column-major
    double* hist;          // cap + 1 residuals
    int* rank;
    double* err;
};
// full-pivot ACA by coupling component, merged into the global pivot order (hsc_aca_comp.cu)
struct AcaComp {
    const double* E;       // coupling, row-major qm x a
    int qm, a, kmax;
    double rtol;
    int ncomp;             // components with at least one coupled column
    const int* row_ptr;    // ncomp + 1
    const int* rows;       // rows of E (12 per body of the component), ascending
    const int* col_ptr;    // ncomp + 1
    const int* cols;       // columns of E (the component's coupled dofs), ascending
    const long long* r_off;// per component: offset of its residual block in Rscratch (when it misses shared memory)
    const int* s_off;      // per component: offset of its step arrays (piv_abs, piv_idx; sums add g)
    const long long* u_off;// per component: offset of its u columns in Ug
    const long long* v_off;// per component: offset of its v columns in Vg
    double* Rscratch;
    double* Ug;
    double* Vg;
    double* piv_abs;
    long long* piv_idx;
    double* sums;          // sum of squares of each component's residual before each step (and after the last)
    int* nsteps;
    int* order;            // 2 x kmax: (component, step) of each global column
    int stot;              // step slots over all components (s_off's total)
    int smem_doubles;
    double* U;             // qm x kmax column-major
    double* V;             // a x kmax column-major
    double* hist;
    int* rank;
    double* err;
};
size_t aca_comp_smem_doubles();
// the warp merge stages every component's step records in shared memory
bool aca_merge_fits(int ncomp, int stot, int kmax);
cudaError_t launch_aca_comp(const AcaComp& p, cudaStream_t st);

size_t aca_cluster_smem_doubles(int m, int nc);
bool aca_cluster_fits(int m, int nc);
cudaError_t launch_aca_cluster(const AcaSys* d_sys, int nsys, size_t smem_doubles, cudaStream_t st);
int aca_cluster_supported(size_t smem_doubles);
// first failed index guard of a self-checking build, per translation unit
void read_fail_aca(long long* out);
void read_fail_pcg(long long* out);
void read_fail_setup(long long* out);

struct GemmArgs {
    const double* A;
    const double* B;
    double* C;
    int M, N, K;
    const int* dM;         // device overrides (rank-dependent sizes), may be null
    const int* dN;
    const int* dK;
    int lda, ldb, ldc;
    int tA, tB;
    double alpha, beta;
};

struct FullSpmv {
    const int* rowptr;
    const int* colidx;
    const double* v64;
    int nnz, n;
    const double* A;       // qm x qm row-major
    const double* E;       // qm x a row-major
    int qm, a;
    const int* act;
    const double* xq;      // qm
    const double* xpad;    // node-padded FEM x
    double* ypad;          // node-padded FEM y
    double* yq;            // qm
    double* rowpart = nullptr;            // qm x abd_row_chunks(a) partials of the ABD rows (null: one warp per row)
    const int* src = nullptr;             // set: read the blocks from the BCOO values through the plan
    const double* bcoo_values = nullptr;  // (column-major 3x3, one triangle) instead of the BSR planes
};

void launch_pattern_hash(const int* rows, const int* cols, long long nnzb, unsigned long long* out, cudaStream_t st);
void launch_fill_bsr(const int* src, const double* values, int nnz, double* v64, float* vf, __nv_bfloat16* vb,
                     cudaStream_t st);
void launch_dinv(int precision, const int* diag_pos, const double* v64, int nnz, int n, void* dinv, int* bad,
                 cudaStream_t st);
void launch_extract(const int* qq, int nqq, const int* qf, int nqf, const double* values, int qm, int a, double* A,
                    double* E, int* node_nz, cudaStream_t st);
cudaError_t launch_aca(const AcaParams& p, int grid, cudaStream_t st);
int aca_blocks_per_sm();
void launch_gemm(const GemmArgs& g, int M, int N, cudaStream_t st);
void launch_cholesky(const double* A, int m, double* L, int* bad, cudaStream_t st);
// P = A^-1 by Cholesky in one CTA; false (nothing launched) when m is too large
// P = A^-1 for an SPD m x m A (dk non-null: only the leading *dk x *dk block, *dk <= m, is
// inverted and written); false when m is too large for the one-CTA kernels
bool launch_chol_inverse(const double* A, int m, double* P, int* bad, cudaStream_t st, const int* dk = nullptr);
// P = A^-1 for an SPD A that is block diagonal over index sets (rows and columns idx[ptr[g] ..
// ptr[g + 1]), every set at most 96): one CTA per set, zeros elsewhere; false if a set is larger
bool launch_inverse_blocks(const double* A, int m, int nblk, int max_blk, const int* ptr, const int* idx, double* P,
                           int* bad, cudaStream_t st);
void launch_chol_solve(const double* L, int m, const double* B, int ldb, double* X, int ldx, int ncol,
                       const int* dncol, double* work, cudaStream_t st);
void launch_ldlt(double* C, int kmax, const int* dk, double* L, double* d, int* bad, cudaStream_t st);
void launch_block12_inverse(const double* A, int qm, double* Binv, int* bad, cudaStream_t st);
void launch_axpby_mat(double* Y, const double* X, double a, double b, int n, int diag_m, double diag_add,
                      cudaStream_t st);
void launch_symmetrize(double* P, int m, cudaStream_t st);
void launch_frob(const double* X, int n, double* out, cudaStream_t st);
void launch_split_rhs(const double* b, int qo, int qm, int fo, int n, const int* perm, double* bq, double* bf,
                      cudaStream_t st);
void launch_wt_vec(const double* W, int qm, int kmax, const int* dk, const double* bq, double* c, cudaStream_t st);
void launch_rhs_lowrank(const double* V, int a, const int* dk, const double* c, const int* act, double* rhs,
                        cudaStream_t st);
void launch_vt_x(const double* V, int a, int kmax, const int* dk, const int* act, const double* x, double* t,
                 cudaStream_t st);
void launch_backsub(const double* P, const double* W, int qm, int kmax, const int* dk, const double* bq,
                    const double* t, double* xq_out, double* xq_copy, cudaStream_t st);
void launch_scatter_x(const double* xpad, int n, int fo, const int* perm, double* xout, cudaStream_t st);
void launch_gather_x(const double* x, int n, int fo, const int* perm, double* xpad, cudaStream_t st);
constexpr int kRowChunk = 1024;  // coupled columns per warp in the ABD rows of the full SpMV
inline int abd_row_chunks(int a) { return a > 0 ? (a + kRowChunk - 1) / kRowChunk : 1; }
void launch_full_spmv(const FullSpmv& f, cudaStream_t st);
void launch_residual(const double* bf, const double* yf, const double* xf, int n, const double* bq, const double* yq,
                     const double* xq, int qm, double* part, int np, double* out, cudaStream_t st);
void launch_scatter_y(const double* ypad, int n, int fo, const int* perm, const double* yq, int qm, int qo, double* y,
                      cudaStream_t st);
void launch_line_step(double* x, const double* d, int N, const double* nd, cudaStream_t st);
void launch_dot2(const double* a, const double* b, const double* c, int N, double* out, cudaStream_t st);
void launch_sub(const double* b, const double* y, double* r, int N, cudaStream_t st);
void launch_gather_rows(const double* src, int a, int k, const int* perm, double* dst, cudaStream_t st);
void launch_split_active_diag(const int* act, int nact_nodes, const int* diag_pos, const double* v64, int nnz,
                              float* vf, __nv_bfloat16* vb, double* dact, cudaStream_t st);
void convert_f64_f32(const double* src, float* dst, long long n, cudaStream_t st);
void set_int(int* p, int v, cudaStream_t st);

}  // namespace hsc
