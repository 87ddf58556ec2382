// C ABI and host orchestration of the B200 HSC solver.
//
// Flow of hsc_solve (the LinearHSC::do_solve of linear_hsc.cu:344-436):
//   analysis (host, once per sparsity pattern): classify BCOO triplets into
//     FEM-FEM / ABD-ABD / ABD-FEM, build the full row-owner BSR plan
//     (sorted columns, source triplet + transpose flag per entry), the
//     sorted active FEM dofs and the per-CTA row partition;
//   numeric (device, no host sync): BSR fill, Dd^-1, A/E extraction, ACA,
//     ABD inverse, W = P U, C = U^T W, C = L D L^T, Vt = V L, rhs;
//   one persistent cooperative PCG launch (hsc_pcg.cu);
//   back-substitution dq = P bq - W V^T x, full residual |b - H x| / |b|;
//   one D2H copy of the per-system scalars, then the status checks of
//   linear_hsc.cu:394-435.
#include <algorithm>
#include <cstdlib>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <functional>
#include <chrono>
#include <thread>
#include <unordered_set>
#include <vector>

#include "../../include/hsc_c_api.h"
#include "hsc_block.cuh"
#include "hsc_learned.cuh"
#include "hsc_partition.h"
#include "hsc_setup.cuh"

using namespace hsc;

namespace {

// Owning device buffer (grow-only).  Move-only: a copy would free the same
// allocation twice when a container of systems reallocates.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), cap(o.cap) { o.p = nullptr; o.cap = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            if (p) cudaFree(p);
            p = o.p; cap = o.cap;
            o.p = nullptr; o.cap = 0;
        }
        return *this;
    }
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t grow(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(bytes, 256));
        if (e == cudaSuccess) cap = std::max<size_t>(bytes, 256);
        return e;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// device scalars of one system, copied to the host once per solve
struct DevScal {
    double pcg[8];            // it, rel, status, normb, nrep (written by the PCG kernel)
    double aca_err;
    double abd_err2;          // |I - A P|_F^2
    double resid[3];          // |b - Hx|^2, |b|^2, b.x
    double nd[2];             // line-search numerator / denominator
    unsigned long long hash;
    int rank;
    int bad_fem;              // FEM diagonal blocks with det <= 0
    int bad_abd;              // non-SPD ABD blocks
    int bad_ldlt;             // zero / non-finite reduced-core pivot
    int pad[4];
    double prev[kPrev];       // record of the previous solve (learned-model features)
    double wl[16];            // learned polynomial weights of this solve
    float feat[kFeat];        // features of this solve
};

struct System {
    // analysis key
    const int* rows = nullptr;
    const int* cols = nullptr;
    long long nnzb = -1;
    int nblock = -1;
    hsc_dof_layout lay{};
    int kmax_for = -1;
    bool analyzed = false;
    unsigned long long hash = 0;
    // sizes
    int n = 0, nnz = 0, a = 0, nqq = 0, nqf = 0, kmax = 0, qm = 0, qo = 0, fo = 0, fn = 0;
    std::vector<int> h_rowptr, h_act, h_colidx, h_rowflag;
    std::vector<int> h_perm, h_iperm, h_part_ptr, h_actp, h_actperm;  // node renumbering, parts, PCG-order active dofs
    bool reordered = false;
    std::vector<int> h_node_body;   // (active node in the caller's order, body) of every coupling block
    bool aca_comp_ok = false;       // the component ACA applies (components of at most 256 rows)
    int ncomp_coupled = 0;
    AcaComp acomp{};
    DevBuf ac_row_ptr, ac_rows, ac_col_ptr, ac_cols, ac_r_off, ac_s_off, ac_u_off, ac_v_off, ac_R, ac_Ug, ac_Vg,
        ac_piv_abs, ac_piv_idx, ac_sums, ac_nsteps, ac_order;
    int ac_stot = 0;
    DevBuf abd_bptr, abd_bidx;  // A's diagonal blocks over coupled bodies (the exact ABD inverse by block)
    int abd_nblk = 0, abd_maxblk = 0;
    // block-local Woodbury preconditioner (hsc_block.cu)
    DevBuf blk_Y, blk_Yact, blk_Vc, blk_pG, blk_G, blk_K, blk_Ka, blk_Kb, blk_pY, blk_pV, blk_pX, blk_pdot, blk_mpub,
        blk_xpub, blk_colof, blk_colptr, blk_cols, blk_bad, blk_C, blk_cta_comp_ptr, blk_cta_comp, blk_cta_comp_slot,
        blk_comp_slot_ptr, blk_comp_of_body, blk_ident, blk_sslice, blk_cslice, blk_cchunk, blk_nloc, blk_slc,
        blk_ssrc, blk_svals, blk_coloff, blk_ctayc;
    BlockPlan blk{};
    int blk_nact_cta = 0;
    // plan
    DevBuf rowptr, colidx, rowid, src, diag_pos, qq, qf, act, ident, rowflag, perm, actp, actperm;
    // numeric
    DevBuf r2;
    DevBuf v64, vf32, vbf16, dinv, A, E, R0, R1, U, V, hist, P, Ptmp, T, term, Binv, L, W, C, Lc, dpiv, vt64, vtmt,
        cvec, tt, ttx, bq, bf, x, r, z, p0, p1, y, t0, t1, node_nz, xq, ypad, yq, work, cg, scal, dact, pact, yact, vt64p,
        zpart, tpart, lcol, rowpart;
    DevBuf dvec[4];           // contiguous-N scratch for refinement
    double h_last[kPrev] = {};   // record of the last solve: 1, lanczos min, max, iterations, q(0)
    double h_prevrec[kPrev] = {};// record the features of the current solve see
    double h_cg[2 * kMaxCoef] = {};
    DevScal h_scal{};
    std::vector<int> h_node_nz;
    std::vector<unsigned short> h_lcol;
    bool aca_on_cluster = false;
};

}  // namespace

struct hsc_ctx {
    hsc_options opt{};
    std::string err;
    int device = 0;
    int num_sms = 148;
    std::vector<System> sys;
    // PCG launch state
    DevBuf d_desc, d_cta_sys, d_cta_row, d_cta_act, d_cta_aidx, d_cta_warp, d_part, d_bar, d_remaining, d_trace;
    DevBuf d_win_off, d_win_nodes, d_win_own, d_win_flag, d_win_act_off, d_win_act;
    int off_z = 0, off_vt = 0, off_y = 0, off_blk = 0, stage_vt = 0, stage_blk = 0;
    int resident = 0, stage_vals = 0, off_wn = 0, off_win = 0, off_val = 0, off_vpc = 0, off_lidx = 0, off_dinv = 0, off_rf = 0;
    int off_own = 0, off_act = 0, own_rows = 0, own_act = 0, off_wflag = 0, off_wact = 0, off_wcorr = 0, wact_max = 0;
    int grid = 0;
    int vt_smem = 0;           // doubles of PCG shared memory after the d.*tt slot
    size_t pcg_smem = 0;       // dynamic shared memory bytes of the PCG launch
    int part_key_gen = -1;
    bool block_layout = false;  // CTA rows = the analysis' parts (the block preconditioner)
    // ACA
    DevBuf aca_psum, aca_pmax, aca_pidx, aca_bar;
    int aca_grid = 0;
    DevBuf d_aca_sys;          // AcaSys descriptors of the systems on the cluster ACA
    int aca_cluster_n = 0;
    size_t aca_cluster_smem = 0;
    int aca_cluster_ok = -1;   // the device can schedule a 16-CTA cluster of the ACA kernel
    DevBuf res_part;
    DevBuf mlp, feat_part;     // learned model (BF16 parameters), feature partials
    bool has_model = false;
    cudaEvent_t ev[9] = {};
    cudaEvent_t ev_blk = nullptr;  // end of the block preconditioner's setup (Y, K) inside the PCG stage
    cudaStream_t side = nullptr;   // the ABD inverses run here, beside the ACA
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_aca = nullptr, ev_pre = nullptr;  // the block setup's start and end on the side stream
    double analysis_ms = 0.0;      // host time of the current call's pattern analysis
    // after a pattern change behind the same pointers, the next solves hash the pattern before they
    // start (one small kernel and a sync) instead of finding out after a full solve
    int pattern_volatile = 0;
    // node partition cache: the last partition and the hash of the adjacency, weights and part count
    // it was made for (a contact change leaves the FEM mesh's pattern, hence its partition, as it was)
    unsigned long long part_hash = 0;
    std::vector<int> part_cache;
    bool stage_events = false;  // record the per-stage events (single system, no graph)
    // graph cache (batch)
    cudaGraphExec_t gexec = nullptr;
    std::vector<const void*> gkey;
    DevScal* h_pinned = nullptr;
    size_t h_pinned_n = 0;
    unsigned char* h_stage = nullptr;  // pinned staging of the per-solve reads (one synchronisation)
    size_t h_stage_bytes = 0;
};

namespace {

constexpr int kResParts = 148;

int fail(hsc_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(ctx, HSC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define GROW(buf, bytes)                                                                        \
    do {                                                                                        \
        cudaError_t e_ = (buf).grow(bytes);                                                     \
        if (e_ != cudaSuccess)                                                                  \
            return fail(ctx, HSC_ERR_ALLOC, std::string("allocation failed: ") + cudaGetErrorString(e_)); \
    } while (0)

size_t vt_bytes(int precision) { return precision == 0 ? sizeof(double) : sizeof(float); }
size_t mt_bytes(int precision) { return precision == 0 ? 8 : (precision == 1 ? 4 : 2); }

int validate_options(const hsc_options* o, std::string& why) {
    if (o->max_rank < 1 || o->max_rank > 256) { why = "max_rank must be in [1, 256]"; return 0; }
    if (o->neumann_order < 1 || o->neumann_order > HSC_MAX_POLY) { why = "neumann_order must be in [1, 16]"; return 0; }
    if (!(o->omega > 0 && o->omega <= 1)) { why = "omega must be in (0, 1]"; return 0; }
    if (o->max_iter < 1) { why = "max_iter must be positive"; return 0; }
    if (!(o->tol >= 0)) { why = "tol must be >= 0"; return 0; }
    if (o->precision < 0 || o->precision > 2) { why = "unknown precision"; return 0; }
    if (o->abd_inverse < 0 || o->abd_inverse > 2) { why = "unknown abd_inverse"; return 0; }
    if (o->preconditioner < HSC_PRECOND_NEUMANN || o->preconditioner > HSC_PRECOND_BLOCK_LEARNED) {
        why = "unknown preconditioner";
        return 0;
    }
    if ((o->preconditioner == HSC_PRECOND_POLY || o->preconditioner == HSC_PRECOND_SCHUR_POLY) &&
        (o->poly_degree < 1 || o->poly_degree > HSC_MAX_POLY)) {
        why = "poly_degree must be in [1, 16]";
        return 0;
    }
    if (o->preconditioner == HSC_PRECOND_BLOCK && (o->poly_degree < 0 || o->poly_degree > HSC_MAX_POLY)) {
        why = "poly_degree must be in [1, 16]";
        return 0;
    }
    if (o->threads_per_row != 0 && o->threads_per_row != 2 && o->threads_per_row != 4 && o->threads_per_row != 8) {
        why = "threads_per_row must be 0 (automatic), 2, 4 or 8";
        return 0;
    }
    if (o->spin_limit < 1000) { why = "spin_limit too small"; return 0; }
    if (!(o->coupled_part_weight >= 1.0 && o->coupled_part_weight <= 8.0)) { why = "coupled_part_weight must be in [1, 8]"; return 0; }
    if (o->graph_replay != 0 && o->graph_replay != 1) { why = "graph_replay must be 0 or 1"; return 0; }
    return 1;
}

// ---------------------------------------------------------------------------
// analysis: sparsity pattern -> plans (host; runs when the pattern changes)
// ---------------------------------------------------------------------------
int analyze(hsc_ctx* ctx, System& S, const hsc_bcoo3& M, const hsc_dof_layout& L, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    if (M.nnzb < 0 || M.nblock <= 0 || M.nnzb >= (1ll << 30)) return fail(ctx, HSC_ERR_INVALID, "bad BCOO sizes");
    if (L.qm < 0 || L.fn <= 0 || L.qm % 12 || L.fn % 3 || L.qo % 3 || L.fo % 3 || L.qm + L.fn != 3 * M.nblock ||
        L.qo < 0 || L.fo < 0 || L.qo + L.qm > 3 * M.nblock || L.fo + L.fn > 3 * M.nblock ||
        (L.qm > 0 && !(L.qo + L.qm <= L.fo || L.fo + L.fn <= L.qo)))
        return fail(ctx, HSC_ERR_INVALID, "HSC requires only ABD (12/body) and FEM (3/node) dofs");  // linear_hsc.cu:199-200
    S.qm = L.qm; S.qo = L.qo; S.fo = L.fo; S.fn = L.fn;
    S.n = L.fn / 3;
    const long long T = M.nnzb;
    std::vector<int> rows(T), cols(T);
    if (T) {
        CK(cudaMemcpyAsync(rows.data(), M.d_rows, sizeof(int) * T, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(cols.data(), M.d_cols, sizeof(int) * T, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    const int qb0 = L.qo / 3, qb1 = (L.qo + L.qm) / 3, fb0 = L.fo / 3, fb1 = (L.fo + L.fn) / 3;
    auto isQ = [&](int b) { return b >= qb0 && b < qb1; };
    auto isF = [&](int b) { return b >= fb0 && b < fb1; };
    std::vector<int> cnt(S.n + 1, 0);
    std::vector<int> qq, qfraw;  // qf raw: t, q, fnode, orient
    std::vector<char> fnode_active(S.n, 0);
    for (long long t = 0; t < T; ++t) {
        const int r = rows[t], c = cols[t];
        if (r < 0 || c < 0 || r >= M.nblock || c >= M.nblock) return fail(ctx, HSC_ERR_INVALID, "block index out of range");
        if (isF(r) && isF(c)) {
            cnt[r - fb0]++;
            if (r != c) cnt[c - fb0]++;
        } else if (isQ(r) && isQ(c)) {
            qq.push_back((int)t); qq.push_back(r - qb0); qq.push_back(c - qb0);
        } else if (isQ(r) && isF(c)) {
            qfraw.push_back((int)t); qfraw.push_back(r - qb0); qfraw.push_back(c - fb0); qfraw.push_back(0);
            fnode_active[c - fb0] = 1;
        } else if (isF(r) && isQ(c)) {
            qfraw.push_back((int)t); qfraw.push_back(c - qb0); qfraw.push_back(r - fb0); qfraw.push_back(1);
            fnode_active[r - fb0] = 1;
        } else {
            return fail(ctx, HSC_ERR_INVALID, "triplet outside the ABD and FEM dof ranges");
        }
    }
    // FEM node renumbering: compact parts of balanced weight, numbered part by part, so that
    // CTA k's contiguous row range is part k (hsc_partition.h).  perm[new] = caller's node.
    {
        std::vector<int> deg(S.n + 1, 0);
        for (long long t = 0; t < T; ++t) {
            const int r = rows[t], c = cols[t];
            if (isF(r) && isF(c) && r != c) { deg[r - fb0]++; deg[c - fb0]++; }
        }
        std::vector<int> aptr(S.n + 1, 0);
        for (int i = 0; i < S.n; ++i) aptr[i + 1] = aptr[i] + deg[i];
        std::vector<int> adj(aptr[S.n]), fillp(aptr.begin(), aptr.end() - 1);
        for (long long t = 0; t < T; ++t) {
            const int r = rows[t], c = cols[t];
            if (isF(r) && isF(c) && r != c) { adj[fillp[r - fb0]++] = c - fb0; adj[fillp[c - fb0]++] = r - fb0; }
        }
        const int nparts = o.reorder ? std::max(1, std::min(ctx->num_sms, S.n / 16)) : 1;
        std::vector<int> part;
        if (nparts > 1) {
            std::vector<double> wgt(S.n);
            for (int i = 0; i < S.n; ++i) wgt[i] = 1.0 + cnt[i];
            const bool blockp = o.preconditioner == HSC_PRECOND_BLOCK || o.preconditioner == HSC_PRECOND_BLOCK_LEARNED;
            const double cw = blockp ? o.coupled_part_weight : 1.0;
            // FNV-1a over (n, parts, adjacency, weights, coupled-part factor): a repeated mesh pattern
            // reuses its partition (also when only the contacts changed)
            unsigned long long h = 1469598103934665603ull;
            auto mix = [&](unsigned long long v) { h = (h ^ v) * 1099511628211ull; };
            mix((unsigned long long)S.n); mix((unsigned long long)nparts);
            for (int i = 0; i <= S.n; ++i) mix((unsigned long long)aptr[i]);
            {  // the adjacency in 16 chunks hashed apart (in parallel), then their hashes in order
                constexpr int kChunks = 16;
                const size_t na = adj.size();
                unsigned long long hc[kChunks];
#pragma omp parallel for schedule(static) if (na >= (1u << 16))
                for (int q = 0; q < kChunks; ++q) {
                    unsigned long long g = 1469598103934665603ull;
                    for (size_t e = na * q / kChunks; e < na * (q + 1) / kChunks; ++e)
                        g = (g ^ (unsigned long long)adj[e]) * 1099511628211ull;
                    hc[q] = g;
                }
                for (int q = 0; q < kChunks; ++q) mix(hc[q]);
            }
            for (int i = 0; i < S.n; ++i) mix((unsigned long long)cnt[i]);
            unsigned long long cwb;
            std::memcpy(&cwb, &cw, sizeof cwb);
            mix(cwb);
            if (ctx->part_hash == h && (int)ctx->part_cache.size() == S.n) {
                part = ctx->part_cache;
            } else {
                part = partition_nodes(S.n, aptr, adj, wgt, nparts);
                if (cw > 1.0) {
                    // the block preconditioner's parts that hold a coupled node also apply their
                    // components' Y columns on every row: their nodes weigh more in a second pass
                    std::vector<char> hot(nparts, 0);
                    for (int i = 0; i < S.n; ++i)
                        if (fnode_active[i]) hot[part[i]] = 1;
                    for (int i = 0; i < S.n; ++i)
                        if (hot[part[i]]) wgt[i] *= cw;
                    part = partition_nodes(S.n, aptr, adj, wgt, nparts);
                }
                ctx->part_hash = h;
                ctx->part_cache = part;
            }
        } else {
            part.assign(S.n, 0);
        }
        S.h_part_ptr.assign(nparts + 1, 0);
        for (int i = 0; i < S.n; ++i) S.h_part_ptr[part[i] + 1]++;
        for (int p = 0; p < nparts; ++p) S.h_part_ptr[p + 1] += S.h_part_ptr[p];
        S.h_perm.assign(S.n, 0);
        S.h_iperm.assign(S.n, 0);
        // inside a part, nodes by decreasing block count (ties by index): rows of similar length sit
        // together, so the 32-row slices of the block preconditioner's layout carry little padding
        // (a counting sort by part keeps the index order inside a part; each part is then sorted
        // stably by block count, in parallel)
        std::vector<int> order(S.n);
        {
            const int np = 1 + *std::max_element(part.begin(), part.end());
            std::vector<int> pstart(np + 1, 0);
            for (int i = 0; i < S.n; ++i) pstart[part[i] + 1]++;
            for (int q = 0; q < np; ++q) pstart[q + 1] += pstart[q];
            std::vector<int> fillq(pstart.begin(), pstart.end() - 1);
            for (int i = 0; i < S.n; ++i) order[fillq[part[i]]++] = i;
#pragma omp parallel for schedule(dynamic, 4) if (np >= 16)
            for (int q = 0; q < np; ++q)
                std::stable_sort(order.begin() + pstart[q], order.begin() + pstart[q + 1],
                                 [&](int x, int y) { return cnt[x] > cnt[y]; });
        }
        for (int ni = 0; ni < S.n; ++ni) {
            S.h_perm[ni] = order[ni];
            S.h_iperm[order[ni]] = ni;
        }
        S.reordered = nparts > 1;
    }
    const std::vector<int>& iperm = S.h_iperm;
    // full BSR plan over the renumbered nodes: rows of D, columns sorted
    S.h_rowptr.assign(S.n + 1, 0);
    for (int i = 0; i < S.n; ++i) S.h_rowptr[i + 1] = S.h_rowptr[i] + cnt[S.h_perm[i]];
    S.nnz = S.h_rowptr[S.n];
    std::vector<int> fillpos(S.h_rowptr.begin(), S.h_rowptr.end() - 1);
    std::vector<long long> ent(S.nnz);  // (col << 32) | packed src
    for (long long t = 0; t < T; ++t) {
        const int r = rows[t], c = cols[t];
        if (isF(r) && isF(c)) {
            const int i = iperm[r - fb0], j = iperm[c - fb0];
            ent[fillpos[i]++] = ((long long)j << 32) | (unsigned)(2 * t);
            if (i != j) ent[fillpos[j]++] = ((long long)i << 32) | (unsigned)(2 * t + 1);
        }
    }
    std::vector<int> colidx(S.nnz), src(S.nnz), diag(S.n, -1);
    int dup_rows = 0;  // rows are independent: sorted in parallel, errors reported after
#pragma omp parallel for schedule(static) reduction(+ : dup_rows) if (S.n >= 4096)
    for (int i = 0; i < S.n; ++i) {
        auto b = ent.begin() + S.h_rowptr[i], e = ent.begin() + S.h_rowptr[i + 1];
        std::sort(b, e);
        for (int k = S.h_rowptr[i]; k < S.h_rowptr[i + 1]; ++k) {
            colidx[k] = (int)(ent[k] >> 32);
            src[k] = (int)(ent[k] & 0xffffffffll);
            if (k > S.h_rowptr[i] && colidx[k] == colidx[k - 1]) ++dup_rows;
            if (colidx[k] == i) diag[i] = k;
        }
    }
    if (dup_rows) return fail(ctx, HSC_ERR_INVALID, "duplicate FEM block (both triangles stored?)");
    for (int i = 0; i < S.n; ++i)
        if (diag[i] < 0) return fail(ctx, HSC_ERR_NONSPD, "HSC: FEM node without a diagonal block");
    // ABD duplicates (both triangles of one pair)
    {
        const int nb = L.qm / 3;
        std::vector<char> seen((size_t)nb * nb, 0);
        for (size_t e = 0; e < qq.size(); e += 3) {
            const int i = std::min(qq[e + 1], qq[e + 2]), j = std::max(qq[e + 1], qq[e + 2]);
            if (seen[(size_t)i * nb + j]) return fail(ctx, HSC_ERR_INVALID, "duplicate ABD block (both triangles stored?)");
            seen[(size_t)i * nb + j] = 1;
        }
    }
    // active FEM nodes (structural) and the coupling list.  The active list keeps the caller's
    // dof order (E's columns, and so the ACA's pivot order, are the reference's); its device copy
    // holds the internal dof numbers.  The PCG sees the same nodes sorted by internal number
    // (actp: each CTA's coupled dofs form one contiguous range), with actperm mapping back.
    std::vector<int> act_index(S.n, -1);
    int nact = 0;
    for (int i = 0; i < S.n; ++i)
        if (fnode_active[i]) act_index[i] = nact++;
    S.a = 3 * nact;
    S.h_act.resize(S.a);
    std::vector<int> act_int(S.a);
    for (int i = 0; i < S.n; ++i)
        if (act_index[i] >= 0)
            for (int c = 0; c < 3; ++c) {
                S.h_act[3 * act_index[i] + c] = 3 * i + c;
                act_int[3 * act_index[i] + c] = 3 * iperm[i] + c;
            }
    S.h_actp.resize(S.a);
    std::vector<int> actperm(S.a);
    std::vector<int> rowflag(S.n, -1);
    {
        int ap = 0;
        for (int ni = 0; ni < S.n; ++ni) {
            const int an = act_index[S.h_perm[ni]];
            if (an < 0) continue;
            rowflag[ni] = ap;
            for (int c = 0; c < 3; ++c) {
                S.h_actp[3 * ap + c] = 3 * ni + c;
                actperm[3 * ap + c] = 3 * an + c;
            }
            ++ap;
        }
    }
    S.h_rowflag = rowflag;
    S.h_actperm = actperm;
    std::vector<int> qf;
    qf.reserve(qfraw.size());
    {
        std::unordered_set<long long> seen;
        for (size_t e = 0; e < qfraw.size(); e += 4) {
            const long long key = (long long)qfraw[e + 1] * S.n + qfraw[e + 2];
            if (!seen.insert(key).second) return fail(ctx, HSC_ERR_INVALID, "duplicate coupling block (both triangles stored?)");
            qf.push_back(qfraw[e]); qf.push_back(qfraw[e + 1]); qf.push_back(act_index[qfraw[e + 2]]); qf.push_back(qfraw[e + 3]);
        }
    }
    S.h_node_body.clear();
    for (size_t e = 0; e < qf.size(); e += 4) { S.h_node_body.push_back(qf[e + 2]); S.h_node_body.push_back(qf[e + 1] / 4); }
    // coupling components for the ACA: bodies joined through the coupled FEM nodes they share
    // (union-find); E is block diagonal over them (rows of their bodies x columns of their nodes)
    std::vector<std::vector<int>> comp_rows, comp_cols;
    {
        const int nbody = S.qm / 12;
        std::vector<int> root(std::max(1, nbody));
        for (int b = 0; b < nbody; ++b) root[b] = b;
        auto find = [&](int b) { while (root[b] != b) { root[b] = root[root[b]]; b = root[b]; } return b; };
        std::vector<int> node_body(std::max(1, nact), -1);
        for (size_t e = 0; e < S.h_node_body.size(); e += 2) {
            const int an = S.h_node_body[e], b = S.h_node_body[e + 1];
            if (node_body[an] < 0) node_body[an] = b;
            else {
                const int ra = find(node_body[an]), rb = find(b);
                if (ra != rb) root[std::max(ra, rb)] = std::min(ra, rb);
            }
        }
        std::vector<int> id(std::max(1, nbody), -1);
        int nc = 0;
        for (int an = 0; an < nact; ++an)   // in order of each component's first coupled node
            if (node_body[an] >= 0 && id[find(node_body[an])] < 0) id[find(node_body[an])] = nc++;
        S.ncomp_coupled = nc;
        comp_rows.assign(nc, {});
        comp_cols.assign(nc, {});
        for (int b = 0; b < nbody; ++b)
            if (id[find(b)] >= 0)
                for (int d = 0; d < 12; ++d) comp_rows[id[find(b)]].push_back(12 * b + d);
        for (int an = 0; an < nact; ++an)
            if (node_body[an] >= 0)
                for (int d = 0; d < 3; ++d) comp_cols[id[find(node_body[an])]].push_back(3 * an + d);
    }
    S.nqq = (int)qq.size() / 3;
    S.nqf = (int)qf.size() / 4;
    // A's blocks: bodies joined by a nonzero body-body block of A (union-find), each block's dofs ascending
    {
        const int nb = S.qm / 12;
        std::vector<int> root(std::max(1, nb));
        for (int b = 0; b < nb; ++b) root[b] = b;
        auto findb = [&](int b) { while (root[b] != b) { root[b] = root[root[b]]; b = root[b]; } return b; };
        for (size_t e = 0; e + 2 < qq.size(); e += 3) {
            const int ra = findb(qq[e + 1] / 4), rb = findb(qq[e + 2] / 4);
            if (ra != rb) root[std::max(ra, rb)] = std::min(ra, rb);
        }
        std::vector<int> gid(std::max(1, nb), -1), bptr(1, 0), bidx;
        std::vector<std::vector<int>> members;
        for (int b = 0; b < nb; ++b) {
            const int r = findb(b);
            if (gid[r] < 0) { gid[r] = (int)members.size(); members.emplace_back(); }
            members[gid[r]].push_back(b);
        }
        S.abd_maxblk = 0;
        for (const auto& mb : members) {
            for (int b : mb)
                for (int d = 0; d < 12; ++d) bidx.push_back(12 * b + d);
            bptr.push_back((int)bidx.size());
            S.abd_maxblk = std::max(S.abd_maxblk, 12 * (int)mb.size());
        }
        S.abd_nblk = (int)members.size();
        if (S.abd_nblk > 0) {
            GROW(S.abd_bptr, sizeof(int) * bptr.size());
            GROW(S.abd_bidx, sizeof(int) * bidx.size());
            CK(cudaMemcpyAsync(S.abd_bptr.p, bptr.data(), sizeof(int) * bptr.size(), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(S.abd_bidx.p, bidx.data(), sizeof(int) * bidx.size(), cudaMemcpyHostToDevice, st));
            CK(cudaStreamSynchronize(st));
        }
    }
    S.kmax = std::min(std::min(o.max_rank, L.qm), S.a);
    // the component ACA's plan
    S.aca_comp_ok = S.kmax > 0 && S.ncomp_coupled > 0;
    for (const auto& r : comp_rows) S.aca_comp_ok = S.aca_comp_ok && r.size() <= 256;
    if (S.aca_comp_ok) {
        int stot = 0;
        for (int g = 0; g < S.ncomp_coupled; ++g)
            stot += std::min(std::min((int)comp_rows[g].size(), (int)comp_cols[g].size()), S.kmax);
        S.aca_comp_ok = aca_merge_fits(S.ncomp_coupled, stot, S.kmax);
    }
    if (S.aca_comp_ok) {
        const int ncg = S.ncomp_coupled;
        std::vector<int> row_ptr(ncg + 1, 0), col_ptr(ncg + 1, 0), rows_all, cols_all, s_off(ncg);
        std::vector<long long> r_off(ncg), u_off(ncg), v_off(ncg);
        long long rtot = 0, utot = 0, vtot = 0;
        int stot = 0;
        for (int g = 0; g < ncg; ++g) {
            const int mr = (int)comp_rows[g].size(), ncl = (int)comp_cols[g].size();
            const int steps = std::min(std::min(mr, ncl), S.kmax);
            rows_all.insert(rows_all.end(), comp_rows[g].begin(), comp_rows[g].end());
            cols_all.insert(cols_all.end(), comp_cols[g].begin(), comp_cols[g].end());
            row_ptr[g + 1] = (int)rows_all.size();
            col_ptr[g + 1] = (int)cols_all.size();
            r_off[g] = rtot; rtot += (long long)mr * ncl;
            u_off[g] = utot; utot += (long long)mr * steps;
            v_off[g] = vtot; vtot += (long long)ncl * steps;
            s_off[g] = stot; stot += steps;
        }
        GROW(S.ac_row_ptr, sizeof(int) * (ncg + 1));
        GROW(S.ac_col_ptr, sizeof(int) * (ncg + 1));
        GROW(S.ac_rows, sizeof(int) * rows_all.size());
        GROW(S.ac_cols, sizeof(int) * cols_all.size());
        GROW(S.ac_r_off, sizeof(long long) * ncg);
        GROW(S.ac_u_off, sizeof(long long) * ncg);
        GROW(S.ac_v_off, sizeof(long long) * ncg);
        GROW(S.ac_s_off, sizeof(int) * ncg);
        GROW(S.ac_R, sizeof(double) * std::max<long long>(1, rtot));
        GROW(S.ac_Ug, sizeof(double) * std::max<long long>(1, utot));
        GROW(S.ac_Vg, sizeof(double) * std::max<long long>(1, vtot));
        GROW(S.ac_piv_abs, sizeof(double) * std::max(1, stot));
        GROW(S.ac_piv_idx, sizeof(long long) * std::max(1, stot));
        GROW(S.ac_sums, sizeof(double) * (stot + ncg));
        GROW(S.ac_nsteps, sizeof(int) * ncg);
        GROW(S.ac_order, sizeof(int) * 2 * S.kmax);
        S.ac_stot = stot;
        CK(cudaMemcpyAsync(S.ac_row_ptr.p, row_ptr.data(), sizeof(int) * (ncg + 1), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_col_ptr.p, col_ptr.data(), sizeof(int) * (ncg + 1), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_rows.p, rows_all.data(), sizeof(int) * rows_all.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_cols.p, cols_all.data(), sizeof(int) * cols_all.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_r_off.p, r_off.data(), sizeof(long long) * ncg, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_u_off.p, u_off.data(), sizeof(long long) * ncg, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_v_off.p, v_off.data(), sizeof(long long) * ncg, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.ac_s_off.p, s_off.data(), sizeof(int) * ncg, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    // ---- device plans and buffers ----
    const int P = o.precision;
    GROW(S.rowptr, sizeof(int) * (S.n + 1));
    GROW(S.colidx, sizeof(int) * std::max(1, S.nnz));
    GROW(S.src, sizeof(int) * std::max(1, S.nnz));
    GROW(S.diag_pos, sizeof(int) * S.n);
    GROW(S.qq, sizeof(int) * std::max<size_t>(3, qq.size()));
    GROW(S.qf, sizeof(int) * std::max<size_t>(4, qf.size()));
    GROW(S.act, sizeof(int) * std::max(1, S.a));
    GROW(S.actp, sizeof(int) * std::max(1, S.a));
    GROW(S.actperm, sizeof(int) * std::max(1, S.a));
    GROW(S.rowflag, sizeof(int) * std::max(1, S.n));
    GROW(S.perm, sizeof(int) * std::max(1, S.n));
    CK(cudaMemcpyAsync(S.rowptr.p, S.h_rowptr.data(), sizeof(int) * (S.n + 1), cudaMemcpyHostToDevice, st));
    {
        std::vector<int> rid(std::max(1, S.nnz));
        for (int i = 0; i < S.n; ++i)
            for (int k = S.h_rowptr[i]; k < S.h_rowptr[i + 1]; ++k) rid[k] = i;
        GROW(S.rowid, sizeof(int) * std::max(1, S.nnz));
        CK(cudaMemcpyAsync(S.rowid.p, rid.data(), sizeof(int) * std::max(1, S.nnz), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    if (S.nnz) {
        CK(cudaMemcpyAsync(S.colidx.p, colidx.data(), sizeof(int) * S.nnz, cudaMemcpyHostToDevice, st));
        S.h_colidx = colidx;
        CK(cudaMemcpyAsync(S.src.p, src.data(), sizeof(int) * S.nnz, cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(S.diag_pos.p, diag.data(), sizeof(int) * S.n, cudaMemcpyHostToDevice, st));
    if (!qq.empty()) CK(cudaMemcpyAsync(S.qq.p, qq.data(), sizeof(int) * qq.size(), cudaMemcpyHostToDevice, st));
    if (!qf.empty()) CK(cudaMemcpyAsync(S.qf.p, qf.data(), sizeof(int) * qf.size(), cudaMemcpyHostToDevice, st));
    if (S.a) {
        CK(cudaMemcpyAsync(S.act.p, act_int.data(), sizeof(int) * S.a, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.actp.p, S.h_actp.data(), sizeof(int) * S.a, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.actperm.p, actperm.data(), sizeof(int) * S.a, cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(S.perm.p, S.h_perm.data(), sizeof(int) * S.n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.rowflag.p, rowflag.data(), sizeof(int) * S.n, cudaMemcpyHostToDevice, st));
    const size_t nz = std::max(1, S.nnz), n4 = 4 * (size_t)std::max(1, S.n), qm = std::max(1, S.qm);
    const size_t km = std::max(1, S.kmax), aa = std::max(1, S.a);
    GROW(S.v64, 9 * sizeof(double) * nz);
    if (P != 0) GROW(S.vf32, 9 * sizeof(float) * nz);
    if (P == 2) GROW(S.vbf16, 9 * sizeof(__nv_bfloat16) * nz);
    GROW(S.dinv, 9 * (P == 0 ? 8 : 4) * (size_t)std::max(1, S.n));
    GROW(S.A, sizeof(double) * qm * qm);
    GROW(S.E, sizeof(double) * qm * aa);
    GROW(S.R0, sizeof(double) * qm * aa);
    GROW(S.R1, sizeof(double) * qm * aa);
    GROW(S.U, sizeof(double) * qm * km);
    GROW(S.V, sizeof(double) * aa * km);
    GROW(S.hist, sizeof(double) * (km + 1));
    GROW(S.P, sizeof(double) * qm * qm);
    GROW(S.Ptmp, sizeof(double) * qm * qm);
    GROW(S.T, sizeof(double) * qm * qm);
    GROW(S.term, sizeof(double) * qm * qm);
    GROW(S.Binv, sizeof(double) * qm * qm);
    GROW(S.L, sizeof(double) * qm * qm);
    GROW(S.ident, sizeof(double) * qm * qm);
    GROW(S.W, sizeof(double) * qm * km);
    GROW(S.C, sizeof(double) * km * km);
    GROW(S.Lc, sizeof(double) * km * km);
    GROW(S.dpiv, sizeof(double) * km);
    GROW(S.vt64, sizeof(double) * aa * km);
    GROW(S.vt64p, sizeof(double) * aa * km);
    GROW(S.cvec, sizeof(double) * km);
    GROW(S.tt, sizeof(double) * 256);
    GROW(S.ttx, sizeof(double) * 256);
    GROW(S.dact, sizeof(double) * 9 * std::max(1, S.a / 3));
    GROW(S.pact, sizeof(double) * aa);
    GROW(S.yact, sizeof(double) * aa);
    GROW(S.bq, sizeof(double) * qm);
    GROW(S.bf, sizeof(double) * n4);
    GROW(S.x, sizeof(double) * n4);
    GROW(S.r, sizeof(double) * n4);
    GROW(S.r2, sizeof(double) * n4);
    GROW(S.z, vt_bytes(P) * n4);
    GROW(S.p0, vt_bytes(P) * n4);
    GROW(S.p1, vt_bytes(P) * n4);
    GROW(S.y, vt_bytes(P) * n4);
    GROW(S.t0, vt_bytes(P) * n4);
    GROW(S.t1, vt_bytes(P) * n4);
    GROW(S.node_nz, sizeof(int) * std::max(1, S.a / 3));
    GROW(S.rowpart, sizeof(double) * std::max(1, S.qm) * abd_row_chunks(S.a));
    GROW(S.xq, sizeof(double) * qm);
    GROW(S.ypad, sizeof(double) * n4);
    GROW(S.yq, sizeof(double) * qm);
    GROW(S.work, sizeof(double) * qm * qm);
    GROW(S.cg, sizeof(double) * 2 * kMaxCoef);
    GROW(S.scal, sizeof(DevScal));
    // contiguous-N vectors; dvec[3] also holds the node-padded x (4 doubles per
    // node) that full_spmv_contig gathers, which is longer than N when n > qm
    const size_t N = std::max(3 * (size_t)M.nblock, n4);
    for (auto& d : S.dvec) GROW(d, sizeof(double) * N);
    if (S.qm) {
        std::vector<double> I((size_t)S.qm * S.qm, 0.0);
        for (int i = 0; i < S.qm; ++i) I[(size_t)i * S.qm + i] = 1.0;
        CK(cudaMemcpyAsync(S.ident.p, I.data(), sizeof(double) * I.size(), cudaMemcpyHostToDevice, st));
    }
    // pattern hash at analysis time
    launch_pattern_hash(M.d_rows, M.d_cols, T, &S.scal.as<DevScal>()->hash, st);
    CK(cudaMemcpyAsync(&S.hash, &S.scal.as<DevScal>()->hash, sizeof(S.hash), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    S.rows = M.d_rows; S.cols = M.d_cols; S.nnzb = M.nnzb; S.nblock = M.nblock; S.lay = L;
    S.kmax_for = (o.max_rank * 16 + o.precision) * 2 + (o.reorder ? 1 : 0);
    S.analyzed = true;
    ctx->part_key_gen = -1;  // CTA partition must be rebuilt
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    return HSC_OK;
}

bool same_key(const System& S, const hsc_bcoo3& M, const hsc_dof_layout& L, const hsc_options& o) {
    return S.analyzed && S.rows == M.d_rows && S.cols == M.d_cols && S.nnzb == M.nnzb && S.nblock == M.nblock &&
           S.lay.qo == L.qo && S.lay.qm == L.qm && S.lay.fo == L.fo && S.lay.fn == L.fn &&
           S.kmax_for == (o.max_rank * 16 + o.precision) * 2 + (o.reorder ? 1 : 0);
}

// ---------------------------------------------------------------------------
// numeric setup (device only, no host sync except the adaptive ABD inverse)
// ---------------------------------------------------------------------------
void gemm(const double* A, int lda, int tA, const double* B, int ldb, int tB, double* C, int ldc, int M, int N, int K,
          double alpha, double beta, cudaStream_t st, const int* dM = nullptr, const int* dN = nullptr,
          const int* dK = nullptr) {
    GemmArgs g{A, B, C, M, N, K, dM, dN, dK, lda, ldb, ldc, tA, tB, alpha, beta};
    launch_gemm(g, M, N, st);
}

int abd_inverse(hsc_ctx* ctx, System& S, cudaStream_t st, bool allow_sync) {
    const hsc_options& o = ctx->opt;
    const int m = S.qm;
    DevScal* ds = S.scal.as<DevScal>();
    double* P = S.P.as<double>();
    if (m == 0) return HSC_OK;
    if (o.abd_inverse == HSC_ABD_EXACT) {
        const bool by_block = S.abd_nblk > 1 &&
                              launch_inverse_blocks(S.A.as<double>(), m, S.abd_nblk, S.abd_maxblk, S.abd_bptr.as<int>(),
                                                    S.abd_bidx.as<int>(), P, &ds->bad_abd, st);
        if (!by_block && !launch_chol_inverse(S.A.as<double>(), m, P, &ds->bad_abd, st)) {
            launch_cholesky(S.A.as<double>(), m, S.L.as<double>(), &ds->bad_abd, st);
            launch_chol_solve(S.L.as<double>(), m, S.ident.as<double>(), m, P, m, m, nullptr, S.work.as<double>(), st);
        }
        launch_symmetrize(P, m, st);
        // |I - A P|_F^2 for the stats
        CK(cudaMemcpyAsync(S.T.p, S.ident.p, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, st));
        gemm(S.A.as<double>(), m, 0, P, m, 0, S.T.as<double>(), m, m, m, m, -1.0, 1.0, st);
        launch_frob(S.T.as<double>(), m * m, &ds->abd_err2, st);
        return HSC_OK;
    }
    // block-Jacobi Neumann (linear_hsc.cu:263-275)
    const double w = o.omega;
    launch_block12_inverse(S.A.as<double>(), m, S.Binv.as<double>(), &ds->bad_abd, st);
    // T = I - w Binv A
    CK(cudaMemcpyAsync(S.T.p, S.ident.p, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, st));
    gemm(S.Binv.as<double>(), m, 0, S.A.as<double>(), m, 0, S.T.as<double>(), m, m, m, m, -w, 1.0, st);
    // term = w Binv, P = term
    CK(cudaMemsetAsync(S.term.p, 0, sizeof(double) * m * m, st));
    launch_axpby_mat(S.term.as<double>(), S.Binv.as<double>(), w, 0.0, m * m, 0, 0.0, st);
    CK(cudaMemcpyAsync(P, S.term.p, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, st));
    for (int k = 1; k < o.neumann_order; ++k) {
        gemm(S.T.as<double>(), m, 0, S.term.as<double>(), m, 0, S.Ptmp.as<double>(), m, m, m, m, 1.0, 0.0, st);
        std::swap(S.term.p, S.Ptmp.p);
        std::swap(S.term.cap, S.Ptmp.cap);
        launch_axpby_mat(P, S.term.as<double>(), 1.0, 1.0, m * m, 0, 0.0, st);
    }
    launch_symmetrize(P, m, st);
    // Rr = I - A P ; err
    auto residual = [&]() {
        cudaMemcpyAsync(S.T.p, S.ident.p, sizeof(double) * m * m, cudaMemcpyDeviceToDevice, st);
        gemm(S.A.as<double>(), m, 0, P, m, 0, S.T.as<double>(), m, m, m, m, -1.0, 1.0, st);
        launch_frob(S.T.as<double>(), m * m, &ds->abd_err2, st);
    };
    residual();
    if (o.abd_inverse != HSC_ABD_ADAPTIVE) return HSC_OK;
    if (!allow_sync) return fail(ctx, HSC_ERR_INVALID, "the adaptive ABD inverse needs host syncs (not graph-capturable)");
    // adaptive doubling P <- P + P (I - A P) (linear_hsc.cu:276-297)
    int d = 0;
    double err2 = 0;
    CK(cudaMemcpyAsync(&err2, &ds->abd_err2, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double err = std::sqrt(err2 / m);
    while (err > o.abd_inverse_tol && d < 48) {
        gemm(P, m, 0, S.T.as<double>(), m, 0, S.Ptmp.as<double>(), m, m, m, m, 1.0, 0.0, st);
        launch_axpby_mat(P, S.Ptmp.as<double>(), 1.0, 1.0, m * m, 0, 0.0, st);
        launch_symmetrize(P, m, st);
        residual();
        CK(cudaMemcpyAsync(&err2, &ds->abd_err2, sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        err = std::sqrt(err2 / m);
        ++d;
        if (!std::isfinite(err)) return fail(ctx, HSC_ERR_NONSPD, "HSC ABD Neumann extension diverged");
    }
    S.h_scal.pcg[7] = d;  // doublings (host side)
    if (err > o.abd_inverse_tol)
        return fail(ctx, HSC_ERR_NONSPD, "HSC ABD inverse residual exceeds abd_inverse_tol after 48 doublings");
    return HSC_OK;
}

void stage_mark(hsc_ctx* ctx, int i, cudaStream_t st) {
    if (ctx->stage_events) cudaEventRecord(ctx->ev[i], st);
}

// numeric setup, part 1: BSR fill, Dd^-1, coupled diagonal blocks, A and E
int numeric_pre(hsc_ctx* ctx, System& S, const hsc_bcoo3& M, cudaStream_t st) {
    const int P = ctx->opt.precision;
    DevScal* ds = S.scal.as<DevScal>();
    S.h_scal.pcg[7] = 0;
    CK(cudaMemsetAsync(ds, 0, offsetof(DevScal, prev), st));  // the previous-solve record stays
    launch_pattern_hash(M.d_rows, M.d_cols, M.nnzb, &ds->hash, st);
    float* vf = P ? S.vf32.as<float>() : nullptr;
    __nv_bfloat16* vb = P == 2 ? S.vbf16.as<__nv_bfloat16>() : nullptr;
    launch_fill_bsr(S.src.as<int>(), M.d_values, S.nnz, S.v64.as<double>(), vf, vb, st);
    launch_dinv(P, S.diag_pos.as<int>(), S.v64.as<double>(), S.nnz, S.n, S.dinv.p, &ds->bad_fem, st);
    launch_split_active_diag(S.actp.as<int>(), S.a / 3, S.diag_pos.as<int>(), S.v64.as<double>(), S.nnz, vf, vb,
                             S.dact.as<double>(), st);
    launch_extract(S.qq.as<int>(), S.nqq, S.qf.as<int>(), S.nqf, M.d_values, S.qm, S.a, S.A.as<double>(),
                   S.E.as<double>(), S.node_nz.as<int>(), st);
    if (S.kmax <= 0) CK(cudaMemsetAsync(&ds->rank, 0, sizeof(int), st));
    return HSC_OK;
}

// ACA of every system's coupling: one cluster launch for the systems whose E
// fits a 16-CTA cluster, the cooperative grid kernel for the others
int aca_all(hsc_ctx* ctx, int count, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    if (ctx->aca_cluster_n > 0) CK(launch_aca_cluster(ctx->d_aca_sys.as<AcaSys>(), ctx->aca_cluster_n,
                                                      ctx->aca_cluster_smem, st));
    for (int s = 0; s < count; ++s) {
        System& S = ctx->sys[s];
        if (S.kmax <= 0 || S.aca_on_cluster) continue;
        DevScal* ds = S.scal.as<DevScal>();
        if (o.aca_components && S.aca_comp_ok) {
            AcaComp& c = S.acomp;
            c.E = S.E.as<double>(); c.qm = S.qm; c.a = S.a; c.kmax = S.kmax;
            c.rtol = o.aca_rtol > 0 ? o.aca_rtol : 0.0;
            c.ncomp = S.ncomp_coupled;
            c.row_ptr = S.ac_row_ptr.as<int>(); c.rows = S.ac_rows.as<int>();
            c.col_ptr = S.ac_col_ptr.as<int>(); c.cols = S.ac_cols.as<int>();
            c.r_off = S.ac_r_off.as<long long>(); c.s_off = S.ac_s_off.as<int>();
            c.u_off = S.ac_u_off.as<long long>(); c.v_off = S.ac_v_off.as<long long>();
            c.Rscratch = S.ac_R.as<double>(); c.Ug = S.ac_Ug.as<double>(); c.Vg = S.ac_Vg.as<double>();
            c.piv_abs = S.ac_piv_abs.as<double>(); c.piv_idx = S.ac_piv_idx.as<long long>();
            c.sums = S.ac_sums.as<double>(); c.nsteps = S.ac_nsteps.as<int>();
            c.order = S.ac_order.as<int>(); c.stot = S.ac_stot;
            c.smem_doubles = (int)aca_comp_smem_doubles();
            c.U = S.U.as<double>(); c.V = S.V.as<double>(); c.hist = S.hist.as<double>();
            c.rank = &ds->rank; c.err = &ds->aca_err;
            CK(launch_aca_comp(c, st));
            continue;
        }
        CK(cudaMemcpyAsync(S.R0.p, S.E.p, sizeof(double) * S.qm * S.a, cudaMemcpyDeviceToDevice, st));
        AcaParams ap{};
        ap.R0 = S.R0.as<double>(); ap.R1 = S.R1.as<double>();
        ap.m = S.qm; ap.nc = S.a; ap.cap = S.kmax; ap.rtol = o.aca_rtol > 0 ? o.aca_rtol : 0.0;
        ap.U = S.U.as<double>(); ap.V = S.V.as<double>(); ap.hist = S.hist.as<double>();
        ap.rank = &ds->rank; ap.err = &ds->aca_err;
        ap.psum = ctx->aca_psum.as<double>(); ap.pmax = ctx->aca_pmax.as<double>(); ap.pidx = ctx->aca_pidx.as<long long>();
        ap.bar = ctx->aca_bar.as<GridBar>(); ap.spin_limit = o.spin_limit;
        CK(cudaMemsetAsync(ctx->aca_bar.p, 0, sizeof(GridBar), st));
        const int grid = ctx->aca_grid;  // upper bound; launch_aca sizes the column strips
        CK(launch_aca(ap, grid, st));
    }
    return HSC_OK;
}

// numeric setup, part 2: ABD inverse P, W = P U, C = U^T W = L D L^T, Vt = V L
// numeric setup, part 2 (after the ACA and the ABD inverse): the reduced core C = U^T P U and its
// LDL^T factors, and (classic PCG) the scaled copy V L_c of V
int numeric_post(hsc_ctx* ctx, System& S, cudaStream_t st) {
    DevScal* ds = S.scal.as<DevScal>();
    if (S.kmax > 0) {
        const int* dk = &ds->rank;
        // W = P U  (qm x k, ld kmax); U column-major (qm x cap) == row-major U^T
        gemm(S.P.as<double>(), S.qm, 0, S.U.as<double>(), S.qm, 1, S.W.as<double>(), S.kmax, S.qm, S.kmax, S.qm,
             1.0, 0.0, st, nullptr, dk, nullptr);
        // C = U^T W (k x k, ld kmax)
        gemm(S.U.as<double>(), S.qm, 0, S.W.as<double>(), S.kmax, 0, S.C.as<double>(), S.kmax, S.kmax, S.kmax, S.qm,
             1.0, 0.0, st, dk, dk, nullptr);
        if (ctx->block_layout && S.blk_C.p)  // the block preconditioner's operator needs C itself
            CK(cudaMemcpyAsync(S.blk_C.p, S.C.p, sizeof(double) * S.kmax * S.kmax, cudaMemcpyDeviceToDevice, st));
        launch_ldlt(S.C.as<double>(), S.kmax, dk, S.Lc.as<double>(), S.dpiv.as<double>(), &ds->bad_ldlt, st);
        if (!ctx->block_layout) {  // the block form applies V C V^T from V and C
            // Vt^T (k x a row-major == Vt column-major a x k) = Lc^T V^T
            CK(cudaMemsetAsync(S.vt64.p, 0, sizeof(double) * S.a * S.kmax, st));
            gemm(S.Lc.as<double>(), S.kmax, 1, S.V.as<double>(), S.a, 0, S.vt64.as<double>(), S.a, S.kmax, S.a,
                 S.kmax, 1.0, 0.0, st, dk, nullptr, dk);
            // the PCG's copy: rows in internal node order (actp)
            launch_gather_rows(S.vt64.as<double>(), S.a, S.kmax, S.actperm.as<int>(), S.vt64p.as<double>(), st);
        }
    }
    stage_mark(ctx, 4, st);
    return HSC_OK;
}

// rhs of the Schur system for right-hand side b (contiguous N)
void schur_rhs(System& S, const double* b, cudaStream_t st) {
    DevScal* ds = S.scal.as<DevScal>();
    launch_split_rhs(b, S.qo, S.qm, S.fo, S.n, S.perm.as<int>(), S.bq.as<double>(), S.bf.as<double>(), st);
    if (S.kmax > 0) {
        launch_wt_vec(S.W.as<double>(), S.qm, S.kmax, &ds->rank, S.bq.as<double>(), S.cvec.as<double>(), st);
        launch_rhs_lowrank(S.V.as<double>(), S.a, &ds->rank, S.cvec.as<double>(), S.act.as<int>(), S.bf.as<double>(), st);
    }
}

// x_out = [dq; dx] after the PCG; also the full residual of (b_orig) if asked
void back_substitute(System& S, const double* b, double* x_out, bool residual, cudaStream_t st) {
    DevScal* ds = S.scal.as<DevScal>();
    // recover the untouched FEM rhs: bf was overwritten by rhs; re-split b
    if (S.kmax > 0)
        launch_vt_x(S.V.as<double>(), S.a, S.kmax, &ds->rank, S.act.as<int>(), S.x.as<double>(), S.cvec.as<double>(), st);
    else
        cudaMemsetAsync(S.cvec.p, 0, sizeof(double) * std::max(1, S.kmax), st);
    launch_split_rhs(b, S.qo, S.qm, S.fo, S.n, S.perm.as<int>(), S.bq.as<double>(), S.bf.as<double>(), st);
    if (S.qm)
        launch_backsub(S.P.as<double>(), S.W.as<double>(), S.qm, std::max(1, S.kmax), &ds->rank, S.bq.as<double>(),
                       S.cvec.as<double>(), x_out + S.qo, S.xq.as<double>(), st);
    launch_scatter_x(S.x.as<double>(), S.n, S.fo, S.perm.as<int>(), x_out, st);
    if (residual) {
        FullSpmv f{S.rowptr.as<int>(), S.colidx.as<int>(), S.v64.as<double>(), S.nnz, S.n, S.A.as<double>(),
                   S.E.as<double>(), S.qm, S.a, S.act.as<int>(), S.xq.as<double>(), S.x.as<double>(),
                   S.ypad.as<double>(), S.yq.as<double>()};
        f.rowpart = S.rowpart.as<double>();
        launch_full_spmv(f, st);
    }
}

// full-system residual dots (after back_substitute with residual=true)
void residual_dots(hsc_ctx* ctx, System& S, cudaStream_t st) {
    DevScal* ds = S.scal.as<DevScal>();
    launch_residual(S.bf.as<double>(), S.ypad.as<double>(), S.x.as<double>(), S.n, S.bq.as<double>(),
                    S.yq.as<double>(), S.xq.as<double>(), S.qm, ctx->res_part.as<double>(), kResParts, ds->resid, st);
}

// y = H x for contiguous N vectors
void full_spmv_contig(System& S, const double* x, double* y, cudaStream_t st, const double* bcoo_values = nullptr) {
    double* xpad = S.dvec[3].as<double>();
    launch_gather_x(x, S.n, S.fo, S.perm.as<int>(), xpad, st);
    if (S.qm) cudaMemcpyAsync(S.xq.p, x + S.qo, sizeof(double) * S.qm, cudaMemcpyDeviceToDevice, st);
    FullSpmv f{S.rowptr.as<int>(), S.colidx.as<int>(), S.v64.as<double>(), S.nnz, S.n, S.A.as<double>(),
               S.E.as<double>(), S.qm, S.a, S.act.as<int>(), S.xq.as<double>(), xpad, S.ypad.as<double>(),
               S.yq.as<double>()};
    f.rowpart = S.rowpart.as<double>();
    if (bcoo_values) { f.src = S.src.as<int>(); f.bcoo_values = bcoo_values; }
    launch_full_spmv(f, st);
    launch_scatter_y(S.ypad.as<double>(), S.n, S.fo, S.perm.as<int>(), S.yq.as<double>(), S.qm, S.qo, y, st);
}

// CTA partition of the persistent launch over the systems in `idx`
int build_partition(hsc_ctx* ctx, const std::vector<int>& idx, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    const size_t smem_cap = 200 * 1024;  // dynamic shared memory budget of one PCG CTA
    const int bps = std::max(1, pcg_blocks_per_sm(o.precision, o.threads_per_row, smem_cap));
    int G = bps * ctx->num_sms;
    const int ns = (int)idx.size();
    if (ns > G) return fail(ctx, HSC_ERR_INVALID, "more systems than co-resident CTAs");
    // Work of a row range in block units: its blocks, one per row (vector updates), and for each node
    // with coupled dofs the low-rank products of every preconditioner term (V^T t partial sums and the
    // V c correction: 2 x 3 dofs x kmax multiply-adds, a block being 9), scaled by a weight that depends
    // on where the CTAs' Vt blocks will live: 0.5 when they fit shared memory (an average block of at most
    // 48 KB; the fastest of 0, 0.5, 1, 2, 4 on the vehicle system), 2 when they stream from L2 (the
    // fastest of 0, 0.5, 2, 3, 4, 8 on the 1 M-tet torus).  HSC_ACTIVE_ROW_WEIGHT overrides it.
    double vt_doubles = 0.0;
    for (int s = 0; s < ns; ++s) {
        const System& S = ctx->sys[idx[s]];
        vt_doubles += (double)S.a * std::max(0, S.kmax);
    }
    double act_w = vt_doubles * sizeof(double) / G <= 48.0 * 1024 ? 0.5 : 2.0;
    if (const char* e = std::getenv("HSC_ACTIVE_ROW_WEIGHT")) act_w = std::max(0.0, std::atof(e));
    std::vector<std::vector<long long>> wpre(ns);  // per system: weighted prefix over rows
    long long tot = 0;
    std::vector<long long> w(ns);
    for (int s = 0; s < ns; ++s) {
        const System& S = ctx->sys[idx[s]];
        const long long extra = (long long)std::llround(act_w * 6.0 * std::max(0, S.kmax) / 9.0);
        auto& pre = wpre[s];
        pre.assign(S.n + 1, 0);
        long long nact_before = 0;
        for (int i = 0; i < S.n; ++i) {
            pre[i] = (long long)S.h_rowptr[i] + i + extra * nact_before;
            if (S.h_rowflag[i] >= 0) ++nact_before;
        }
        pre[S.n] = (long long)S.h_rowptr[S.n] + S.n + extra * nact_before;
        w[s] = std::max<long long>(1, pre[S.n]);
        tot += w[s];
    }
    // CTAs per system proportional to work, at least one, at most one per 16 rows
    std::vector<int> nc(ns);
    int used = 0;
    for (int s = 0; s < ns; ++s) {
        const System& S = ctx->sys[idx[s]];
        int want = (int)std::floor((double)G * w[s] / tot);
        want = std::max(1, std::min(want, std::max(1, S.n / 16)));
        nc[s] = want;
        used += want;
    }
    while (used > G) {
        int big = (int)(std::max_element(nc.begin(), nc.end()) - nc.begin());
        nc[big]--; used--;
    }
    G = used;
    std::vector<int> cta_sys(G), cta_row(2 * G), cta_act(2 * G), cta_aidx(G, -1);
    std::vector<SysDesc> desc(ns);
    int c = 0;
    for (int s = 0; s < ns; ++s) {
        System& S = ctx->sys[idx[s]];
        const int b = c;
        const auto& pre = wpre[s];
        const long long rows_w = pre[S.n];
        int row = 0;
        // the analysis' parts, when the block preconditioner asks for one CTA per part, else a
        // weighted split of the rows (it also weighs the coupled rows' low-rank work)
        const bool by_part = ctx->block_layout && (int)S.h_part_ptr.size() == nc[s] + 1 && nc[s] > 1;
        for (int k = 0; k < nc[s]; ++k, ++c) {
            const long long target = rows_w * (k + 1) / nc[s];
            const int rb = row;
            if (k == nc[s] - 1) row = S.n;
            else if (by_part) row = S.h_part_ptr[k + 1];
            else
                while (row < S.n && pre[row] < target) ++row;
            cta_sys[c] = s;
            cta_row[2 * c] = rb;
            cta_row[2 * c + 1] = row;
            cta_act[2 * c] = (int)(std::lower_bound(S.h_actp.begin(), S.h_actp.end(), 3 * rb) - S.h_actp.begin());
            cta_act[2 * c + 1] = (int)(std::lower_bound(S.h_actp.begin(), S.h_actp.end(), 3 * row) - S.h_actp.begin());
        }
        SysDesc& d = desc[s];
        d.n = S.n; d.nnz = S.nnz; d.a = S.a; d.kmax = S.kmax; d.cta_begin = b; d.cta_end = c;
        d.rowptr = S.rowptr.as<int>(); d.colidx = S.colidx.as<int>(); d.rowid = S.rowid.as<int>();
        d.vals = o.precision ? S.vf32.p : S.v64.p;
        d.vals_pc = o.precision == 2 ? S.vbf16.p : d.vals;
        d.vals64 = S.v64.as<double>(); d.dinv = S.dinv.p;
        d.act = S.actp.as<int>(); d.rowflag = S.rowflag.as<int>(); d.dact = S.dact.as<double>();
        d.vt64 = S.vt64p.as<double>(); d.dpiv = S.dpiv.as<double>(); d.rank = &S.scal.as<DevScal>()->rank;
        d.pact = S.pact.as<double>(); d.yact = S.yact.as<double>(); d.ttx = S.ttx.as<double>();
        GROW(S.zpart, sizeof(double) * std::max(1, S.kmax) * (size_t)(c - b));
        d.zpart = S.zpart.as<double>();
        int nact = 0;
        for (int k = b; k < c; ++k)
            if (cta_act[2 * k + 1] > cta_act[2 * k]) cta_aidx[k] = nact++;
        d.nact_cta = nact;
        GROW(S.tpart, sizeof(double) * 2 * std::max(1, S.kmax) * (size_t)std::max(1, nact));
        d.tpart = S.tpart.as<double>();
        d.wdev = o.preconditioner == HSC_PRECOND_LEARNED ? S.scal.as<DevScal>()->wl : nullptr;
        d.x = S.x.as<double>(); d.r = S.r.as<double>(); d.r2 = S.r2.as<double>(); d.rhs = S.bf.as<double>(); d.z = S.z.p;
        d.p[0] = S.p0.p; d.p[1] = S.p1.p; d.y = S.y.p; d.t[0] = S.t0.p; d.t[1] = S.t1.p; d.tt = S.tt.as<double>();
        d.out = S.scal.as<DevScal>()->pcg; d.cg_coef = S.cg.as<double>(); d.max_coef = kMaxCoef;
    }
    // warp-owned row ranges: kWarps + 1 boundaries per CTA, balanced by blocks
    std::vector<int> cta_warp((size_t)(kWarps + 1) * G);
    int Zmax = 0, VTmax = 0, Rmax = 0, BLKmax = 0;
    for (int k = 0; k < G; ++k) {
        const System& S = ctx->sys[idx[cta_sys[k]]];
        const int rb = cta_row[2 * k], re = cta_row[2 * k + 1];
        const long long kb0 = S.h_rowptr[rb], nb = (long long)S.h_rowptr[re] - kb0;
        int row = rb;
        for (int w = 0; w <= kWarps; ++w) {
            if (w == kWarps) row = re;
            else {
                const long long target = kb0 + nb * w / kWarps;
                while (row < re && S.h_rowptr[row] < target) ++row;
            }
            cta_warp[(size_t)(kWarps + 1) * k + w] = row;
        }
        const int na = cta_act[2 * k + 1] - cta_act[2 * k];
        Zmax = std::max(Zmax, (na + 1) & ~1);
        VTmax = std::max(VTmax, na * std::max(0, S.kmax));
        Rmax = std::max(Rmax, re - rb);
        BLKmax = std::max(BLKmax, (int)nb);
    }
    // vector windows (resident mode): the sorted nodes each CTA's blocks read,
    // and per BSR entry the window position of its column
    std::vector<int> win_off(G + 1, 0), win_nodes, win_own(G, 0), win_flag, win_act_off(G + 1, 0), win_act;
    int Wmax = 0, WAmax = 0;
    bool win_ok = o.resident != 0;
    if (win_ok) {
        // each CTA's window on its own (in parallel; per-thread node stamps), then concatenated
        int maxn = 1;
        for (int k = 0; k < G; ++k) {
            System& S = ctx->sys[idx[cta_sys[k]]];
            maxn = std::max(maxn, S.n);
            if (S.h_lcol.size() != (size_t)S.nnz) S.h_lcol.assign(S.nnz, 0);
        }
        std::vector<std::vector<int>> wl(G);
        int too_big = 0;
#pragma omp parallel reduction(+ : too_big) if (G >= 16)
        {
            std::vector<int> stamp(maxn, -1), pos(maxn, 0);
#pragma omp for schedule(dynamic, 4)
            for (int k = 0; k < G; ++k) {
                System& S = ctx->sys[idx[cta_sys[k]]];
                const int rb = cta_row[2 * k], re = cta_row[2 * k + 1];
                const int kb0 = S.h_rowptr[rb], kb1 = S.h_rowptr[re];
                std::vector<int>& w = wl[k];
                for (int e = kb0; e < kb1; ++e) {
                    const int c = S.h_colidx[e];
                    if (stamp[c] != k) { stamp[c] = k; w.push_back(c); }
                }
                std::sort(w.begin(), w.end());
                for (int i = 0; i < (int)w.size(); ++i) pos[w[i]] = i;
                if (w.size() > 65535 || re - rb > 65535) { ++too_big; continue; }
                for (int e = kb0; e < kb1; ++e) S.h_lcol[e] = (unsigned short)pos[S.h_colidx[e]];
                win_own[k] = rb < re ? pos[rb] : 0;
            }
        }
        if (too_big) win_ok = false;
        for (int k = 0; k < G && win_ok; ++k) {
            System& S = ctx->sys[idx[cta_sys[k]]];
            const std::vector<int>& w = wl[k];
            win_off[k + 1] = win_off[k] + (int)w.size();
            win_nodes.insert(win_nodes.end(), w.begin(), w.end());
            int nwa = 0;
            for (int c : w) {
                const int an = S.h_rowflag[c];
                win_flag.push_back(an >= 0 ? nwa : -1);
                if (an >= 0) { win_act.push_back(an); ++nwa; }
            }
            win_act_off[k + 1] = win_act_off[k] + nwa;
            WAmax = std::max(WAmax, nwa);
            Wmax = std::max(Wmax, (int)w.size());
        }
    }
    // shared-memory layout (doubles).  Resident when the BSR slice, its indices
    // and the window fit next to the rest; otherwise staging of the Vt blocks
    // and of the column indices is dropped (in that order) when the budget does
    // not hold them
    const int budget = (int)(smem_cap / sizeof(double));
    // the kernel's static shared memory (parameter block, system descriptor, three k-vectors of
    // kMaxRank doubles, warp scratch: about 7.5 KB) comes out of the same 227 KB
    const int res_budget = (int)((227 * 1024 - 8 * 1024) / sizeof(double));
    const int base = kMaxRank + Zmax + 3 * Rmax + 2;
    if (base > budget) return fail(ctx, HSC_ERR_INVALID, "too many rows or coupled dofs in one CTA");
    const size_t vtb = vt_bytes(o.precision), mtb = o.precision == 0 ? 8 : 4;
    auto dbl = [](size_t bytes) { return (int)((bytes + 15) / 16 * 2); };  // 16-byte aligned, in doubles
    const int W_wn = dbl(sizeof(int) * (size_t)Wmax), W_win = dbl(4 * vtb * (size_t)Wmax);
    const int W_val = dbl(9 * mtb * (size_t)BLKmax), W_vpc = o.precision == 2 ? dbl(9 * 2 * (size_t)BLKmax) : 0;
    const int W_lidx = dbl(4 * (size_t)BLKmax);
    const int W_dinv = dbl(9 * mtb * (size_t)Rmax), W_rf = dbl(sizeof(int) * (2 * (size_t)Rmax + 1));
    const int W_own = dbl(2 * 3 * 8 * (size_t)Rmax + 4 * 3 * vtb * (size_t)Rmax);
    const int W_act = dbl(2 * 8 * (size_t)Zmax + sizeof(int) * (size_t)Zmax);
    const int W_wflag = dbl(sizeof(int) * (size_t)Wmax), W_wact = dbl(sizeof(int) * (size_t)WAmax);
    const int W_wcorr = dbl(3 * 8 * (size_t)WAmax);
    const int res_need = base + 4 + W_wn + W_win + W_val + W_vpc + W_lidx + W_dinv + W_rf + W_own + W_act + W_wflag +
                         W_wact + W_wcorr;
    // resident: Vt blocks first (they sit on the critical path of the coupled
    // CTAs), then the value planes; without room for the planes they stream
    const int need_novals = res_need - W_val - W_vpc;
    int stage_vt = 1, stage_blk = 1, resident = 0, stage_vals = 0;
    if (win_ok && need_novals <= res_budget) {
        resident = 1;
        stage_blk = 0;
        if (res_need + VTmax <= res_budget) { stage_vt = 1; stage_vals = 1; }
        else if (need_novals + VTmax <= res_budget) { stage_vt = 1; stage_vals = 0; }
        else if (res_need <= res_budget) { stage_vt = 0; stage_vals = 1; }
        else { stage_vt = 0; stage_vals = 0; }
    } else if (base + VTmax + BLKmax > budget) {
        if (base + BLKmax <= budget) stage_vt = 0;
        else if (base + VTmax <= budget) stage_blk = 0;
        else { stage_vt = 0; stage_blk = 0; }
    }
    ctx->off_z = kMaxRank;
    ctx->off_vt = ctx->off_z + Zmax;
    ctx->off_y = ctx->off_vt + (stage_vt ? VTmax : 0);
    ctx->off_y += ctx->off_y & 1;
    ctx->off_blk = ctx->off_y + 3 * Rmax + 1;
    ctx->off_blk += ctx->off_blk & 1;
    ctx->stage_vt = stage_vt;
    ctx->stage_blk = stage_blk;
    ctx->vt_smem = Zmax + VTmax;
    ctx->resident = resident;
    ctx->stage_vals = stage_vals;
    if (resident) {
        ctx->off_wn = ctx->off_blk;
        ctx->off_win = ctx->off_wn + W_wn;
        ctx->off_val = ctx->off_win + W_win;
        ctx->off_vpc = ctx->off_val + (stage_vals ? W_val : 0);
        ctx->off_lidx = ctx->off_vpc + (stage_vals ? W_vpc : 0);
        ctx->off_dinv = ctx->off_lidx + W_lidx;
        ctx->off_rf = ctx->off_dinv + W_dinv;
        ctx->off_own = ctx->off_rf + W_rf;
        ctx->off_act = ctx->off_own + W_own;
        ctx->own_rows = Rmax;
        ctx->own_act = Zmax;
        ctx->off_wflag = ctx->off_act + W_act;
        ctx->off_wact = ctx->off_wflag + W_wflag;
        ctx->off_wcorr = ctx->off_wact + W_wact;
        ctx->wact_max = WAmax;
        ctx->pcg_smem = sizeof(double) * (size_t)(ctx->off_wcorr + W_wcorr);
        GROW(ctx->d_win_flag, sizeof(int) * std::max<size_t>(1, win_flag.size()));
        GROW(ctx->d_win_act_off, sizeof(int) * (G + 1));
        GROW(ctx->d_win_act, sizeof(int) * std::max<size_t>(1, win_act.size()));
        if (!win_flag.empty())
            CK(cudaMemcpyAsync(ctx->d_win_flag.p, win_flag.data(), sizeof(int) * win_flag.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->d_win_act_off.p, win_act_off.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
        if (!win_act.empty())
            CK(cudaMemcpyAsync(ctx->d_win_act.p, win_act.data(), sizeof(int) * win_act.size(), cudaMemcpyHostToDevice, st));
        GROW(ctx->d_win_off, sizeof(int) * (G + 1));
        GROW(ctx->d_win_nodes, sizeof(int) * std::max<size_t>(1, win_nodes.size()));
        GROW(ctx->d_win_own, sizeof(int) * G);
        CK(cudaMemcpyAsync(ctx->d_win_off.p, win_off.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
        if (!win_nodes.empty())
            CK(cudaMemcpyAsync(ctx->d_win_nodes.p, win_nodes.data(), sizeof(int) * win_nodes.size(),
                               cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->d_win_own.p, win_own.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
        for (int s2 = 0; s2 < ns; ++s2) {
            System& S = ctx->sys[idx[s2]];
            GROW(S.lcol, sizeof(unsigned short) * (size_t)std::max(1, S.nnz));
            if (S.nnz)
                CK(cudaMemcpyAsync(S.lcol.p, S.h_lcol.data(), sizeof(unsigned short) * S.nnz, cudaMemcpyHostToDevice, st));
            desc[s2].lcol = S.lcol.as<unsigned short>();
        }
    } else {
        ctx->pcg_smem = sizeof(double) * (size_t)(ctx->off_blk + (stage_blk ? BLKmax : 0));
    }
    GROW(ctx->d_cta_warp, sizeof(int) * cta_warp.size());
    CK(cudaMemcpyAsync(ctx->d_cta_warp.p, cta_warp.data(), sizeof(int) * cta_warp.size(), cudaMemcpyHostToDevice, st));
    GROW(ctx->d_desc, sizeof(SysDesc) * ns);
    GROW(ctx->d_cta_sys, sizeof(int) * G);
    GROW(ctx->d_cta_row, sizeof(int) * 2 * G);
    GROW(ctx->d_cta_act, sizeof(int) * 2 * G);
    GROW(ctx->d_cta_aidx, sizeof(int) * G);
    GROW(ctx->d_part, sizeof(double) * 3 * G);
    if (!ctx->d_bar.p) {
        GROW(ctx->d_bar, sizeof(GridBar));
        CK(cudaMemsetAsync(ctx->d_bar.p, 0, sizeof(GridBar), st));
    }
    GROW(ctx->d_remaining, sizeof(int));
    CK(cudaMemcpyAsync(ctx->d_desc.p, desc.data(), sizeof(SysDesc) * ns, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cta_sys.p, cta_sys.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cta_row.p, cta_row.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cta_act.p, cta_act.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->d_cta_aidx.p, cta_aidx.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
    // cluster-ACA descriptors (pointers only: valid for every numeric pass of this analysis)
    std::vector<AcaSys> aca;
    size_t aca_smem = 0;
    for (int s2 = 0; s2 < ns; ++s2) {
        System& S = ctx->sys[idx[s2]];
        S.aca_on_cluster = false;
        if (S.kmax <= 0 || !o.aca_cluster || !aca_cluster_fits(S.qm, S.a)) continue;
        if (o.aca_components && S.aca_comp_ok) continue;  // the component ACA serves it
        const size_t need = aca_cluster_smem_doubles(S.qm, S.a);
        if (ctx->aca_cluster_ok < 0) ctx->aca_cluster_ok = aca_cluster_supported(25600) > 0 ? 1 : 0;
        if (!ctx->aca_cluster_ok) continue;
        DevScal* ds = S.scal.as<DevScal>();
        aca.push_back(AcaSys{S.E.as<double>(), S.qm, S.a, S.kmax, o.aca_rtol > 0 ? o.aca_rtol : 0.0,
                             S.U.as<double>(), S.V.as<double>(), S.hist.as<double>(), &ds->rank, &ds->aca_err});
        aca_smem = std::max(aca_smem, need);
        S.aca_on_cluster = true;
    }
    ctx->aca_cluster_n = (int)aca.size();
    ctx->aca_cluster_smem = aca_smem;
    if (!aca.empty()) {
        GROW(ctx->d_aca_sys, sizeof(AcaSys) * aca.size());
        CK(cudaMemcpyAsync(ctx->d_aca_sys.p, aca.data(), sizeof(AcaSys) * aca.size(), cudaMemcpyHostToDevice, st));
    }
    CK(cudaStreamSynchronize(st));  // host vectors die here
    ctx->grid = G;
    return HSC_OK;
}

int launch_pcg_all(hsc_ctx* ctx, int nsys, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    PcgParams prm{};
    prm.sys = ctx->d_desc.as<SysDesc>();
    prm.nsys = nsys;
    prm.cta_sys = ctx->d_cta_sys.as<int>();
    prm.cta_row = ctx->d_cta_row.as<int>();
    prm.cta_act = ctx->d_cta_act.as<int>();
    prm.cta_aidx = ctx->d_cta_aidx.as<int>();
    prm.part_rr = ctx->d_part.as<double>();
    prm.part_rz = ctx->d_part.as<double>() + ctx->grid;
    prm.part_pap = ctx->d_part.as<double>() + 2 * ctx->grid;
    prm.vt_smem = ctx->vt_smem;
    prm.cta_warp = ctx->d_cta_warp.as<int>();
    prm.off_z = ctx->off_z; prm.off_vt = ctx->off_vt; prm.off_y = ctx->off_y; prm.off_blk = ctx->off_blk;
    prm.stage_vt = ctx->stage_vt; prm.stage_blk = ctx->stage_blk;
    prm.resident = ctx->resident;
    prm.stage_vals = ctx->stage_vals;
    prm.win_off = ctx->d_win_off.as<int>(); prm.win_nodes = ctx->d_win_nodes.as<int>(); prm.win_own = ctx->d_win_own.as<int>();
    prm.off_wn = ctx->off_wn; prm.off_win = ctx->off_win; prm.off_val = ctx->off_val; prm.off_vpc = ctx->off_vpc;
    prm.off_lidx = ctx->off_lidx;
    prm.off_dinv = ctx->off_dinv; prm.off_rf = ctx->off_rf;
    prm.off_own = ctx->off_own; prm.off_act = ctx->off_act; prm.own_rows = ctx->own_rows; prm.own_act = ctx->own_act;
    prm.win_flag = ctx->d_win_flag.as<int>(); prm.win_act_off = ctx->d_win_act_off.as<int>();
    prm.win_act = ctx->d_win_act.as<int>();
    prm.off_wflag = ctx->off_wflag; prm.off_wact = ctx->off_wact; prm.off_wcorr = ctx->off_wcorr;
    prm.wact_max = ctx->wact_max;
    prm.trace = nullptr;
    prm.trace_iters = 0;
    if (o.trace_iterations > 0) {
        const size_t nt = (size_t)ctx->grid * o.trace_iterations * kTraceEvents;
        GROW(ctx->d_trace, sizeof(unsigned long long) * nt);
        CK(cudaMemsetAsync(ctx->d_trace.p, 0, sizeof(unsigned long long) * nt, st));
        prm.trace = ctx->d_trace.as<unsigned long long>();
        prm.trace_iters = o.trace_iterations;
    }
    prm.bar = ctx->d_bar.as<GridBar>();
    prm.remaining = ctx->d_remaining.as<int>();
    prm.omega = o.omega;
    prm.schur_basis = o.preconditioner == HSC_PRECOND_SCHUR_POLY || o.preconditioner == HSC_PRECOND_LEARNED;
    if (o.preconditioner == HSC_PRECOND_POLY || o.preconditioner == HSC_PRECOND_SCHUR_POLY) {
        prm.nterms = o.poly_degree;
        for (int k = 0; k < o.poly_degree; ++k) prm.w[k] = o.poly_weights[k];
    } else if (o.preconditioner == HSC_PRECOND_LEARNED) {
        prm.nterms = kPolyOut;                 // weights from the device (SysDesc::wdev)
        for (int k = 0; k < kPolyOut; ++k) prm.w[k] = 1.0;
    } else {
        prm.nterms = o.neumann_order;
        for (int k = 0; k < o.neumann_order; ++k) prm.w[k] = 1.0;
    }
    prm.fuse = ctx->resident && o.fuse_update && !prm.schur_basis && prm.nterms >= 2;
    prm.tol = o.tol;
    prm.max_iter = o.max_iter;
    prm.rr_every = o.residual_replacement;
    prm.spin_limit = o.spin_limit;
    // the barrier counter grows by one per CTA and grid barrier (at most nterms + 2 per iteration,
    // one iteration more for the replacement slot) and keeps its top bit for the abort flag
    if ((double)(o.max_iter + 2) * (prm.nterms + 3) * ctx->grid >= (double)kBarAbortBit)
        return fail(ctx, HSC_ERR_INVALID, "max_iter too large for the grid barrier counter");
    CK(cudaMemsetAsync(ctx->d_bar.p, 0, sizeof(GridBar), st));
    set_int(ctx->d_remaining.as<int>(), nsys, st);
    // automatic tile width: 4 on the shared-memory-resident path, 2 when the slices stream from memory
    // (the 1 M-tet torus: 5-7 % less time per iteration than 4; the vehicle system: 4 is fastest)
    const int tpr = o.threads_per_row ? o.threads_per_row : (ctx->resident ? 4 : 2);
    CK(launch_pcg(o.precision, tpr, prm, ctx->grid, ctx->pcg_smem, st));
    return HSC_OK;
}

// ---------------------------------------------------------------------------
// block-local Woodbury preconditioner: the static plan (coupling components,
// their contributor CTAs, shared-memory layout) after build_partition laid the
// CTAs on the analysis' parts, and the per-solve launches
// ---------------------------------------------------------------------------
int build_block_plan(hsc_ctx* ctx, System& S, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    if (!ctx->resident || ctx->grid < 1) return fail(ctx, HSC_ERR_INVALID, "the block preconditioner needs the resident CTA windows");
    const int G = ctx->grid;
    // cta rows / coupled ranges as build_partition placed them
    std::vector<int> cta_row(2 * G), cta_act(2 * G), cta_aidx(G), win_off(G + 1), win_own(G);
    CK(cudaMemcpyAsync(win_own.data(), ctx->d_win_own.p, sizeof(int) * G, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(cta_row.data(), ctx->d_cta_row.p, sizeof(int) * 2 * G, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(cta_act.data(), ctx->d_cta_act.p, sizeof(int) * 2 * G, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(cta_aidx.data(), ctx->d_cta_aidx.p, sizeof(int) * G, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(win_off.data(), ctx->d_win_off.p, sizeof(int) * (G + 1), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // coupling components: bodies joined through the FEM nodes they share (union-find)
    const int nbody = S.qm / 12;
    std::vector<int> root(std::max(1, nbody));
    for (int b = 0; b < nbody; ++b) root[b] = b;
    std::function<int(int)> find = [&](int b) { while (root[b] != b) { root[b] = root[root[b]]; b = root[b]; } return b; };
    const int nact_nodes = S.a / 3;
    std::vector<int> node_first_body(std::max(1, nact_nodes), -1);
    for (size_t e = 0; e < S.h_node_body.size(); e += 2) {
        const int an = S.h_node_body[e], b = S.h_node_body[e + 1];
        if (node_first_body[an] < 0) node_first_body[an] = b;
        else {
            const int ra = find(node_first_body[an]), rb = find(b);
            if (ra != rb) root[std::max(ra, rb)] = std::min(ra, rb);
        }
    }
    std::vector<int> comp_of_body(std::max(1, nbody), 0);
    std::vector<int> comp_id(std::max(1, nbody), -1);
    int ncomp = 0;
    for (int b = 0; b < nbody; ++b) {
        const int r = find(b);
        if (comp_id[r] < 0) comp_id[r] = ncomp++;
        comp_of_body[b] = comp_id[r];
    }
    if (ncomp > 256) return fail(ctx, HSC_ERR_INVALID, "the block preconditioner supports at most 256 coupling components");
    // per CTA: the components of its coupled nodes (actp order), and each component's contributor CTAs
    std::vector<std::vector<int>> comps(G);
    for (int c = 0; c < G; ++c) {
        std::vector<int> cs;
        for (int i = cta_act[2 * c]; i < cta_act[2 * c + 1]; i += 3) {
            const int b = node_first_body[S.h_actperm[i] / 3];
            if (b >= 0) cs.push_back(comp_of_body[b]);
        }
        std::sort(cs.begin(), cs.end());
        cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
        comps[c] = cs;
    }
    std::vector<int> comp_slot_ptr(ncomp + 1, 0);
    for (int c = 0; c < G; ++c)
        for (int g : comps[c]) comp_slot_ptr[g + 1]++;
    for (int g = 0; g < ncomp; ++g) comp_slot_ptr[g + 1] += comp_slot_ptr[g];
    std::vector<int> fill(comp_slot_ptr.begin(), comp_slot_ptr.end() - 1);
    std::vector<int> cta_comp_ptr(G + 1, 0), cta_comp, cta_comp_slot;
    for (int c = 0; c < G; ++c) {
        for (int g : comps[c]) { cta_comp.push_back(g); cta_comp_slot.push_back(fill[g]++); }
        cta_comp_ptr[c + 1] = (int)cta_comp.size();
    }
    const int nslot = comp_slot_ptr[ncomp];
    // columns a component can hold: 12 per body, 3 per coupled node, the rank cap
    std::vector<int> comp_bodies(ncomp, 0), comp_nodes(ncomp, 0), comp_cap(ncomp, 0);
    for (int b = 0; b < nbody; ++b) comp_bodies[comp_of_body[b]]++;
    for (int an = 0; an < nact_nodes; ++an)
        if (node_first_body[an] >= 0) comp_nodes[comp_of_body[node_first_body[an]]]++;
    for (int g = 0; g < ncomp; ++g) comp_cap[g] = std::min(std::min(12 * comp_bodies[g], 3 * comp_nodes[g]), S.kmax);
    int NCOL = 1;
    for (int c = 0; c < G; ++c) {
        int nc = 0;
        for (int g : comps[c]) nc += comp_cap[g];
        NCOL = std::max(NCOL, std::min(nc, std::max(1, S.kmax)));
    }
    int nact_cta = 0;
    for (int c = 0; c < G; ++c) nact_cta += cta_aidx[c] >= 0;
    // maxima for the shared-memory layout
    int R = 1, W = 1, NA = 1;
    for (int c = 0; c < G; ++c) {
        const int rb = cta_row[2 * c], re = cta_row[2 * c + 1];
        R = std::max(R, re - rb);
        W = std::max(W, win_off[c + 1] - win_off[c]);
        NA = std::max(NA, cta_act[2 * c + 1] - cta_act[2 * c]);
    }
    if (R > kBlockMaxRows)
        return fail(ctx, HSC_ERR_INVALID, "a part of the block preconditioner has more rows than one CTA holds");
    if (S.h_lcol.size() != (size_t)S.nnz)
        return fail(ctx, HSC_ERR_INVALID, "the block preconditioner needs the CTA windows of the BSR entries");
    // sliced ELL of each CTA's rows: slices of kSliceRows rows; a row's slots are its diagonal block,
    // its blocks whose column lies in the part (ascending), the others (ascending), then padding to
    // the slice's even width; lane 2 r + h of chunk c holds slot 2 c + h of the slice's row r
    std::vector<int4> sslice;
    std::vector<int> cslice(G + 1, 0), cchunk(G + 1, 0), ssrc;
    std::vector<unsigned short> nloc(std::max(1, S.n), 0), slc;
    int NS = 1, NCH = 1;
    {
        // each CTA's slices on their own (in parallel), then concatenated in CTA order
        std::vector<std::vector<int4>> c_slice(G);
        std::vector<std::vector<int>> c_src(G);
        std::vector<std::vector<unsigned short>> c_lc(G);
        int not_contig = 0;
#pragma omp parallel reduction(+ : not_contig) if (G >= 16)
        {
            std::vector<std::vector<int>> rowslots(kSliceRows);
#pragma omp for schedule(dynamic, 4)
            for (int c = 0; c < G; ++c) {
                const int rb = cta_row[2 * c], re = cta_row[2 * c + 1];
                int ch_rel = 0;
                for (int r0 = rb; r0 < re; r0 += kSliceRows) {
                    const int r1 = std::min(re, r0 + kSliceRows);
                    int width = 0, lwidth = 0, lmin = 1 << 30;
                    for (int r = r0; r < r1; ++r) {
                        std::vector<int>& sl = rowslots[r - r0];
                        sl.clear();
                        int diag = -1;
                        for (int e = S.h_rowptr[r]; e < S.h_rowptr[r + 1]; ++e)
                            if (S.h_colidx[e] == r) diag = e;
                        sl.push_back(diag);
                        for (int e = S.h_rowptr[r]; e < S.h_rowptr[r + 1]; ++e) {
                            const int col = S.h_colidx[e];
                            if (col >= rb && col < re && S.h_lcol[e] != win_own[c] + (col - rb)) ++not_contig;
                            if (col != r && col >= rb && col < re) sl.push_back(e);
                        }
                        nloc[r] = (unsigned short)sl.size();
                        for (int e = S.h_rowptr[r]; e < S.h_rowptr[r + 1]; ++e) {
                            const int col = S.h_colidx[e];
                            if (col < rb || col >= re) sl.push_back(e);
                        }
                        width = std::max(width, (int)sl.size());
                        lwidth = std::max(lwidth, (int)nloc[r]);
                        lmin = std::min(lmin, (int)nloc[r]);
                    }
                    const int nch = (width + 1) / 2;
                    // chunks holding a local slot of some row: [0, (lwidth + 1) / 2); a remote one: [lmin / 2, nch)
                    c_slice[c].push_back(make_int4(ch_rel, nch, (lwidth + 1) / 2, lmin / 2));
                    const size_t base = c_src[c].size();
                    c_src[c].resize(base + (size_t)32 * nch, -1);
                    c_lc[c].resize(base + (size_t)32 * nch, (unsigned short)win_own[c]);
                    for (int r = r0; r < r1; ++r) {
                        const std::vector<int>& sl = rowslots[r - r0];
                        for (int j = 0; j < (int)sl.size(); ++j) {
                            const size_t at = base + (size_t)32 * (j / 2) + 2 * (r - r0) + (j & 1);
                            c_src[c][at] = sl[j];
                            c_lc[c][at] = sl[j] >= 0 ? S.h_lcol[sl[j]] : (unsigned short)win_own[c];
                        }
                    }
                    ch_rel += nch;
                }
            }
        }
        if (not_contig) return fail(ctx, HSC_ERR_INVALID, "a part's rows are not contiguous in its window");
        for (int c = 0; c < G; ++c) {
            sslice.insert(sslice.end(), c_slice[c].begin(), c_slice[c].end());
            ssrc.insert(ssrc.end(), c_src[c].begin(), c_src[c].end());
            slc.insert(slc.end(), c_lc[c].begin(), c_lc[c].end());
            const int ch_rel = (int)(c_src[c].size() / 32);
            cslice[c + 1] = (int)sslice.size();
            cchunk[c + 1] = cchunk[c] + ch_rel;
            NS = std::max(NS, cslice[c + 1] - cslice[c]);
            NCH = std::max(NCH, ch_rel);
        }
    }
    const long long nchunk = cchunk[G];
    const int km = std::max(1, S.kmax);
    const size_t n4 = 4 * (size_t)std::max(1, S.n);
    GROW(S.blk_Y, sizeof(float) * km * n4);
    GROW(S.blk_Yact, sizeof(double) * std::max(1, S.a) * km);
    GROW(S.blk_Vc, sizeof(double) * std::max(1, S.a) * km);
    GROW(S.blk_pG, sizeof(double) * std::max(1, nact_cta) * km * km);
    GROW(S.blk_G, sizeof(double) * km * km);
    GROW(S.blk_K, sizeof(double) * km * km);
    GROW(S.blk_Ka, sizeof(double) * km * km);
    GROW(S.blk_Kb, sizeof(double) * km * km);
    GROW(S.blk_C, sizeof(double) * km * km);
    GROW(S.blk_pY, sizeof(double) * std::max(1, nslot) * km);
    GROW(S.blk_pV, sizeof(double) * std::max(1, nslot) * km);
    GROW(S.blk_pX, sizeof(double) * std::max(1, nslot) * km);
    GROW(S.blk_pdot, sizeof(double) * 4 * G);
    GROW(S.blk_mpub, sizeof(double) * n4);
    GROW(S.blk_xpub, sizeof(double) * n4);
    GROW(S.blk_colof, sizeof(int) * km);
    GROW(S.blk_colptr, sizeof(int) * (ncomp + 1));
    GROW(S.blk_cols, sizeof(int) * km);
    GROW(S.blk_coloff, sizeof(int) * (km + 1));
    GROW(S.blk_bad, sizeof(int) * 4);
    GROW(S.blk_cta_comp_ptr, sizeof(int) * (G + 1));
    GROW(S.blk_cta_comp, sizeof(int) * std::max<size_t>(1, cta_comp.size()));
    GROW(S.blk_cta_comp_slot, sizeof(int) * std::max<size_t>(1, cta_comp_slot.size()));
    GROW(S.blk_comp_slot_ptr, sizeof(int) * (ncomp + 1));
    GROW(S.blk_comp_of_body, sizeof(int) * std::max(1, nbody));
    GROW(S.blk_sslice, sizeof(int4) * std::max<size_t>(1, sslice.size()));
    GROW(S.blk_cslice, sizeof(int) * (G + 1));
    GROW(S.blk_cchunk, sizeof(int) * (G + 1));
    GROW(S.blk_nloc, sizeof(unsigned short) * nloc.size());
    GROW(S.blk_slc, sizeof(unsigned short) * std::max<size_t>(1, slc.size()));
    GROW(S.blk_ssrc, sizeof(int) * std::max<size_t>(1, ssrc.size()));
    GROW(S.blk_svals, (o.precision ? sizeof(float) : sizeof(double)) * kChunkVals * std::max<long long>(1, nchunk));
    if (!sslice.empty())
        CK(cudaMemcpyAsync(S.blk_sslice.p, sslice.data(), sizeof(int4) * sslice.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.blk_cslice.p, cslice.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.blk_cchunk.p, cchunk.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(S.blk_nloc.p, nloc.data(), sizeof(unsigned short) * nloc.size(), cudaMemcpyHostToDevice, st));
    if (!slc.empty()) {
        CK(cudaMemcpyAsync(S.blk_slc.p, slc.data(), sizeof(unsigned short) * slc.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.blk_ssrc.p, ssrc.data(), sizeof(int) * ssrc.size(), cudaMemcpyHostToDevice, st));
    }
    if (S.blk_ident.cap < sizeof(double) * km * km) {
        GROW(S.blk_ident, sizeof(double) * km * km);
        std::vector<double> I((size_t)km * km, 0.0);
        for (int i = 0; i < km; ++i) I[(size_t)i * km + i] = 1.0;
        CK(cudaMemcpyAsync(S.blk_ident.p, I.data(), sizeof(double) * I.size(), cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
    }
    CK(cudaMemcpyAsync(S.blk_cta_comp_ptr.p, cta_comp_ptr.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
    if (!cta_comp.empty()) {
        CK(cudaMemcpyAsync(S.blk_cta_comp.p, cta_comp.data(), sizeof(int) * cta_comp.size(), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(S.blk_cta_comp_slot.p, cta_comp_slot.data(), sizeof(int) * cta_comp_slot.size(),
                           cudaMemcpyHostToDevice, st));
    }
    CK(cudaMemcpyAsync(S.blk_comp_slot_ptr.p, comp_slot_ptr.data(), sizeof(int) * (ncomp + 1), cudaMemcpyHostToDevice, st));
    if (nbody)
        CK(cudaMemcpyAsync(S.blk_comp_of_body.p, comp_of_body.data(), sizeof(int) * nbody, cudaMemcpyHostToDevice, st));
    BlockPlan& b = S.blk;
    b = BlockPlan{};
    b.n = S.n; b.nnz = S.nnz; b.a = S.a; b.kmax = km; b.qm = S.qm;
    b.rank = &S.scal.as<DevScal>()->rank;
    b.vals = o.precision ? S.vf32.p : S.v64.p;
    b.dinv = S.dinv.p;
    b.dact = o.precision ? S.dact.as<double>() : nullptr;
    b.rowflag = S.rowflag.as<int>(); b.actp = S.actp.as<int>(); b.actperm = S.actperm.as<int>();
    b.V = S.V.as<double>(); b.C = S.blk_C.as<double>(); b.Lc = S.Lc.as<double>(); b.dpiv = S.dpiv.as<double>();
    b.U = S.U.as<double>();
    b.K = S.blk_K.as<double>(); b.Ka = S.blk_Ka.as<double>(); b.Kb = S.blk_Kb.as<double>();
    b.Y = S.blk_Y.as<float>(); b.Yact = S.blk_Yact.as<double>(); b.Vc = S.blk_Vc.as<double>();
    b.pG = S.blk_pG.as<double>(); b.G = S.blk_G.as<double>();
    b.bad = S.blk_bad.as<int>();
    b.ident = S.blk_ident.as<double>();
    b.G_ctas = G;
    b.cta_row = ctx->d_cta_row.as<int>(); b.cta_act = ctx->d_cta_act.as<int>(); b.cta_aidx = ctx->d_cta_aidx.as<int>();
    b.win_off = ctx->d_win_off.as<int>(); b.win_nodes = ctx->d_win_nodes.as<int>(); b.win_own = ctx->d_win_own.as<int>();
    b.sell_slice = S.blk_sslice.as<int4>(); b.cta_slice = S.blk_cslice.as<int>(); b.cta_chunk = S.blk_cchunk.as<int>();
    b.sell_nloc = S.blk_nloc.as<unsigned short>(); b.sell_lc = S.blk_slc.as<unsigned short>();
    b.sell_src = S.blk_ssrc.as<int>(); b.sell_vals = S.blk_svals.p; b.nchunk = nchunk;
    b.ncomp = ncomp;
    b.comp_of_body = S.blk_comp_of_body.as<int>();
    b.cta_comp_ptr = S.blk_cta_comp_ptr.as<int>(); b.cta_comp = S.blk_cta_comp.as<int>();
    b.cta_comp_slot = S.blk_cta_comp_slot.as<int>(); b.comp_slot_ptr = S.blk_comp_slot_ptr.as<int>();
    b.nslot = nslot;
    b.comp_of_col = S.blk_colof.as<int>(); b.comp_col_ptr = S.blk_colptr.as<int>(); b.comp_cols = S.blk_cols.as<int>();
    b.col_off = S.blk_coloff.as<int>();
    b.x = S.x.as<double>(); b.rhs = S.bf.as<double>(); b.mpub = S.blk_mpub.as<double>(); b.xpub = S.blk_xpub.as<double>();
    b.pY = S.blk_pY.as<double>(); b.pV = S.blk_pV.as<double>(); b.pX = S.blk_pX.as<double>(); b.pdot = S.blk_pdot.as<double>();
    b.bar = ctx->d_bar.as<GridBar>();
    b.out = S.scal.as<DevScal>()->pcg;
    b.cg_coef = S.cg.as<double>(); b.max_coef = kMaxCoef;
    b.R = R; b.NS = NS; b.NCH = NCH; b.W = W; b.NA = NA; b.NCOL = NCOL;
    // stage the value planes when they fit; then each CTA stages as many of its Y columns (3 R
    // floats each) as fit after its own value chunks
    const size_t cap = (size_t)block_max_smem();
    bool vals_in = block_smem_bytes(o.precision, b, true) <= cap && b.smem_y <= cap;
    block_smem_bytes(o.precision, b, vals_in);
    if (std::max(b.smem, b.smem_y) > cap)
        return fail(ctx, HSC_ERR_INVALID, "a part of the block preconditioner does not fit one CTA's shared memory");
    {
        const size_t mt = o.precision ? sizeof(float) : sizeof(double);
        std::vector<int> yc(2 * G);
        size_t need = b.smem;
        int nyc_max = 0;
        for (int c = 0; c < G; ++c) {
            const size_t off = b.off_val + (vals_in ? (mt * kChunkVals * (size_t)(cchunk[c + 1] - cchunk[c]) + 15) / 16 * 16 : 0);
            const size_t col = sizeof(float) * 3 * (size_t)std::max(1, cta_row[2 * c + 1] - cta_row[2 * c]);
            int ncap = 0;
            for (int g : comps[c]) ncap += comp_cap[g];
            ncap = std::min(ncap, km);
            const int nyc = off < cap ? (int)std::min<size_t>((size_t)ncap, (cap - off) / col) : 0;
            yc[2 * c] = (int)off;
            yc[2 * c + 1] = nyc;
            need = std::max(need, off + col * nyc);
            nyc_max = std::max(nyc_max, nyc);
        }
        GROW(S.blk_ctayc, sizeof(int) * 2 * G);
        CK(cudaMemcpyAsync(S.blk_ctayc.p, yc.data(), sizeof(int) * 2 * G, cudaMemcpyHostToDevice, st));
        CK(cudaStreamSynchronize(st));
        b.cta_yc = S.blk_ctayc.as<int>();
        b.NYC = nyc_max;
        b.smem = need;
    }
    S.blk_nact_cta = nact_cta;
    return HSC_OK;
}

// the block setup that needs only the ACA's factors: the sliced-ELL values, the components'
// columns, Y = L V with the V^T Y partials, and their sum G; it runs on the side stream beside the
// reduced core and the Schur rhs.  Also sets the plan's polynomial and PCG controls.
int launch_block_pre(hsc_ctx* ctx, System& S, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    BlockPlan& b = S.blk;
    const bool learned = o.preconditioner == HSC_PRECOND_BLOCK_LEARNED;
    if (learned) {
        b.nterms = kPolyOut;
        b.wdev = S.scal.as<DevScal>()->wl;
        for (int k = 0; k < kPolyOut; ++k) b.w[k] = 1.0;
    } else {
        b.wdev = nullptr;
        b.nterms = o.poly_degree > 0 ? o.poly_degree : o.neumann_order;
        for (int k = 0; k < b.nterms; ++k) b.w[k] = o.poly_degree > 0 ? o.poly_weights[k] : 1.0;
    }
    b.omega = o.omega;
    b.tol = o.tol;
    b.max_iter = o.max_iter;
    b.rr_every = o.residual_replacement;
    b.spin_limit = o.spin_limit;
    // grid barriers: two per iteration, two more per true-residual check
    if ((double)(o.max_iter + 4) * 4 * b.G_ctas >= (double)kBarAbortBit)
        return fail(ctx, HSC_ERR_INVALID, "max_iter too large for the grid barrier counter");
    launch_block_fill(o.precision, b, st);
    if (S.kmax > 0) {
        launch_block_columns(b, st);
        CK(launch_block_y(o.precision, b, st));
        launch_block_g(b, S.blk_nact_cta, st);
    } else {
        CK(cudaMemsetAsync(S.blk_colptr.p, 0, sizeof(int) * (b.ncomp + 1), st));
    }
    return HSC_OK;
}

// the Woodbury core K (needs the reduced core's LDL^T factors) and the PCG
int launch_block_solve(hsc_ctx* ctx, System& S, cudaStream_t st) {
    const hsc_options& o = ctx->opt;
    BlockPlan& b = S.blk;
    if (S.kmax > 0) launch_block_k(b, st);
    if (ctx->stage_events) CK(cudaEventRecord(ctx->ev_blk, st));
    b.trace = nullptr;
    b.trace_iters = 0;
    if (o.trace_iterations > 0) {
        const size_t nt = (size_t)b.G_ctas * o.trace_iterations * kTraceEvents;
        GROW(ctx->d_trace, sizeof(unsigned long long) * nt);
        CK(cudaMemsetAsync(ctx->d_trace.p, 0, sizeof(unsigned long long) * nt, st));
        b.trace = ctx->d_trace.as<unsigned long long>();
        b.trace_iters = o.trace_iterations;
    }
    CK(cudaMemsetAsync(ctx->d_bar.p, 0, sizeof(GridBar), st));
    CK(launch_block_pcg(o.precision, b, st));
    return HSC_OK;
}

// extreme Ritz values of the CG Lanczos tridiagonal (bisection on Sturm counts)
void lanczos_extremes(const double* coef, int m, double& lo, double& hi) {
    lo = hi = 0.0;
    std::vector<double> d, e;
    for (int i = 0; i < m; ++i) {
        const double a = coef[2 * i];
        if (!(a > 0) || !std::isfinite(a)) break;
        double di = 1.0 / a;
        if (i > 0) {
            const double bprev = coef[2 * (i - 1) + 1], aprev = coef[2 * (i - 1)];
            if (!(bprev > 0)) break;
            di += bprev / aprev;
            e.push_back(std::sqrt(bprev) / aprev);
        }
        d.push_back(di);
    }
    const int n = (int)d.size();
    if (n == 0) return;
    if ((int)e.size() > n - 1) e.resize(n - 1);
    double gl = 1e300, gu = -1e300;
    for (int i = 0; i < n; ++i) {
        double rad = (i > 0 ? std::fabs(e[i - 1]) : 0) + (i < n - 1 ? std::fabs(e[i]) : 0);
        gl = std::min(gl, d[i] - rad);
        gu = std::max(gu, d[i] + rad);
    }
    // both extremes at once, each bracket quartered per pass: six independent Sturm counts share one
    // walk down the diagonal (their divisions overlap), to a relative width of 1e-12
    std::vector<double> e2(std::max(1, n - 1));
    for (int i = 0; i + 1 < n; ++i) e2[i] = e[i] * e[i];
    double a[2] = {gl, gl}, b[2] = {gu, gu};
    const int kk[2] = {0, n - 1};
    for (int it = 0; it < 100; ++it) {
        bool done[2];
        for (int t = 0; t < 2; ++t) done[t] = !(b[t] - a[t] > 1e-12 * std::max(std::fabs(a[t]), std::fabs(b[t])));
        if (done[0] && done[1]) break;
        double x[6], q[6];
        int c[6];
        for (int t = 0; t < 2; ++t)
            for (int p = 0; p < 3; ++p) x[3 * t + p] = a[t] + (b[t] - a[t]) * 0.25 * (p + 1);
        for (int j = 0; j < 6; ++j) { q[j] = d[0] - x[j]; c[j] = q[j] < 0; }
        for (int i = 1; i < n; ++i)
            for (int j = 0; j < 6; ++j) {
                if (q[j] == 0) q[j] = 1e-300;
                q[j] = d[i] - x[j] - e2[i - 1] / q[j];
                c[j] += q[j] < 0;
            }
        for (int t = 0; t < 2; ++t) {
            if (done[t]) continue;
            const int k = kk[t];  // the bracket keeps the k-th eigenvalue: count(lower) <= k < count(upper)
            if (c[3 * t] > k) b[t] = x[3 * t];
            else if (c[3 * t + 1] > k) { a[t] = x[3 * t]; b[t] = x[3 * t + 1]; }
            else if (c[3 * t + 2] > k) { a[t] = x[3 * t + 1]; b[t] = x[3 * t + 2]; }
            else a[t] = x[3 * t + 2];
        }
    }
    lo = 0.5 * (a[0] + b[0]);
    hi = 0.5 * (a[1] + b[1]);
}

void fill_stats(hsc_ctx* ctx, System& S, const DevScal& h, hsc_stats* out, bool residual, int refinement_steps,
                int total_iters) {
    const hsc_options& o = ctx->opt;
    hsc_stats s{};
    s.fem_dofs = S.fn;
    s.abd_dofs = S.qm;
    int nzn = 0;
    for (int v : S.h_node_nz) nzn += v != 0;
    s.active_fem_dofs = 3 * nzn;
    s.rank = h.rank;
    s.pcg_iterations = total_iters >= 0 ? total_iters : (int)h.pcg[0];
    s.neumann_doublings = (int)S.h_scal.pcg[7];
    s.refinement_steps = refinement_steps;
    s.precision = o.precision;
    s.preconditioner = o.preconditioner;
    s.residual_replacements = (int)h.pcg[4];
    s.aca_relative_error = h.aca_err;
    s.schur_relative_residual = h.pcg[1];
    s.abd_inverse_residual = S.qm ? std::sqrt(h.abd_err2 / S.qm) : 0.0;
    s.full_residual_limit = o.full_residual_limit;
    s.nnzb = S.nnzb;
    if (residual) {
        s.full_relative_residual = h.resid[1] > 0 ? std::sqrt(h.resid[0] / h.resid[1]) : 0.0;
        s.descent = h.resid[2];
    } else {
        s.full_relative_residual = NAN;
        s.descent = NAN;
    }
    *out = s;
}

// status of one system from its scalars (the asserts of linear_hsc.cu)
int system_status(hsc_ctx* ctx, const System& S, const DevScal& h, bool residual, int grid_abort, std::string& msg) {
    const hsc_options& o = ctx->opt;
    char buf[256];
    if (h.bad_fem) { snprintf(buf, sizeof buf, "HSC: %d non-positive FEM diagonal blocks", h.bad_fem); msg = buf; return HSC_ERR_NONSPD; }
    if (h.bad_abd) { msg = "HSC: non-SPD ABD block"; return HSC_ERR_NONSPD; }
    if (h.bad_ldlt) { msg = "HSC: singular reduced core U^T P U"; return HSC_ERR_NONSPD; }
    if (h.aca_err < 0) { msg = "HSC: the ACA cluster launch did not get 16 CTAs"; return HSC_ERR_CUDA; }
    const int st = (int)h.pcg[2];
    if (grid_abort || st < 0) { msg = "HSC: a device-side wait gave up (grid barrier timeout)"; return HSC_ERR_TIMEOUT; }
    if (st == 3) { snprintf(buf, sizeof buf, "HSC Schur PCG breakdown at iteration %d. No fallback.", (int)h.pcg[0]); msg = buf; return HSC_ERR_BREAKDOWN; }
    if (st == 4) { snprintf(buf, sizeof buf, "HSC Schur PCG did not converge: iterations=%d, residual=%g", (int)h.pcg[0], h.pcg[1]); msg = buf; return HSC_ERR_NOCONV; }
    if (residual) {
        const double bn2 = h.resid[1];
        const double full = bn2 > 0 ? std::sqrt(h.resid[0] / bn2) : 0.0;
        if (!(std::isfinite(h.resid[2]) && (h.resid[2] > 0 || bn2 == 0))) { msg = "HSC returned a non-descent direction"; return HSC_ERR_NONDESCENT; }
        if (!(std::isfinite(full) && full <= o.full_residual_limit)) {
            snprintf(buf, sizeof buf, "HSC full-system residual %g exceeds %g. No fallback.", full, o.full_residual_limit);
            msg = buf;
            return HSC_ERR_RESIDUAL;
        }
    }
    return HSC_OK;
}

int ensure_common(hsc_ctx* ctx, cudaStream_t st) {
    GROW(ctx->aca_psum, sizeof(double) * 4096);
    GROW(ctx->aca_pmax, sizeof(double) * 4096);
    GROW(ctx->aca_pidx, sizeof(long long) * 4096);
    if (!ctx->aca_bar.p) {
        GROW(ctx->aca_bar, sizeof(GridBar));
        CK(cudaMemsetAsync(ctx->aca_bar.p, 0, sizeof(GridBar), st));  // read back even when no grid ACA ran
    }
    GROW(ctx->res_part, sizeof(double) * 3 * kResParts);
    GROW(ctx->feat_part, sizeof(double) * kFeatParts * 2 * std::max(1, ctx->num_sms));
    if (!ctx->aca_grid) ctx->aca_grid = std::min(4096, std::max(1, aca_blocks_per_sm()) * ctx->num_sms);
    if (!ctx->ev[0]) {
        for (auto& e : ctx->ev) CK(cudaEventCreate(&e));
        CK(cudaEventCreate(&ctx->ev_blk));
        CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ev_aca, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ctx->ev_pre, cudaEventDisableTiming));
        CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    }
    (void)st;
    return HSC_OK;
}

int read_scalars(hsc_ctx* ctx, const std::vector<int>& idx, cudaStream_t st, int& grid_abort) {
    if (ctx->h_pinned_n < idx.size()) {
        if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
        ctx->h_pinned = nullptr;
        CK(cudaMallocHost((void**)&ctx->h_pinned, sizeof(DevScal) * idx.size()));
        ctx->h_pinned_n = idx.size();
    }
    // everything else of this read goes through one pinned staging buffer as well: copies into
    // pageable memory would each wait for their own round trip
    size_t need = 2 * sizeof(GridBar);
    for (size_t s = 0; s < idx.size(); ++s) {
        const System& S = ctx->sys[idx[s]];
        need += sizeof(double) * 2 * kMaxCoef + ((sizeof(int) * (S.a / 3) + 7) & ~(size_t)7);
    }
    if (ctx->h_stage_bytes < need) {
        if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->h_stage_bytes = 0;
        CK(cudaMallocHost((void**)&ctx->h_stage, need));
        ctx->h_stage_bytes = need;
    }
    for (size_t s = 0; s < idx.size(); ++s)
        CK(cudaMemcpyAsync(ctx->h_pinned + s, ctx->sys[idx[s]].scal.p, sizeof(DevScal), cudaMemcpyDeviceToHost, st));
    GridBar* gbs = reinterpret_cast<GridBar*>(ctx->h_stage);
    gbs[0] = GridBar{};
    gbs[1] = GridBar{};
    if (ctx->d_bar.p) CK(cudaMemcpyAsync(&gbs[0], ctx->d_bar.p, sizeof(GridBar), cudaMemcpyDeviceToHost, st));
    if (ctx->aca_bar.p) CK(cudaMemcpyAsync(&gbs[1], ctx->aca_bar.p, sizeof(GridBar), cudaMemcpyDeviceToHost, st));
    size_t off = 2 * sizeof(GridBar);
    std::vector<size_t> offs(idx.size());
    for (size_t s = 0; s < idx.size(); ++s) {
        System& S = ctx->sys[idx[s]];
        offs[s] = off;
        if (S.cg.p)
            CK(cudaMemcpyAsync(ctx->h_stage + off, S.cg.p, sizeof(double) * 2 * kMaxCoef, cudaMemcpyDeviceToHost, st));
        off += sizeof(double) * 2 * kMaxCoef;
        if (S.a)
            CK(cudaMemcpyAsync(ctx->h_stage + off, S.node_nz.p, sizeof(int) * (S.a / 3), cudaMemcpyDeviceToHost, st));
        off += (sizeof(int) * (S.a / 3) + 7) & ~(size_t)7;
    }
    CK(cudaStreamSynchronize(st));
    grid_abort = gbs[0].abort | gbs[1].abort;
    for (size_t s = 0; s < idx.size(); ++s) {
        System& S = ctx->sys[idx[s]];
        const double d7 = S.h_scal.pcg[7];
        S.h_scal = ctx->h_pinned[s];
        S.h_scal.pcg[7] = d7;
        if (S.cg.p) std::memcpy(S.h_cg, ctx->h_stage + offs[s], sizeof(double) * 2 * kMaxCoef);
        S.h_node_nz.resize(S.a / 3);
        if (S.a)
            std::memcpy(S.h_node_nz.data(), ctx->h_stage + offs[s] + sizeof(double) * 2 * kMaxCoef,
                        sizeof(int) * (S.a / 3));
    }
    return HSC_OK;
}

FeatArgs feat_args(hsc_ctx* ctx, System& S, bool with_model) {
    DevScal* ds = S.scal.as<DevScal>();
    FeatArgs f{};
    f.n = S.n; f.nnz = S.nnz; f.a = S.a; f.kmax = S.kmax;
    f.rowptr = S.rowptr.as<int>(); f.colidx = S.colidx.as<int>(); f.diag_pos = S.diag_pos.as<int>();
    f.rowflag = S.rowflag.as<int>(); f.v64 = S.v64.as<double>(); f.rank = &ds->rank;
    f.vt64 = S.vt64p.as<double>(); f.dpiv = S.dpiv.as<double>(); f.prev = ds->prev;
    f.mlp = with_model ? ctx->mlp.as<uint16_t>() : nullptr;
    f.feat = ds->feat; f.w = ds->wl;
    f.part = ctx->feat_part.as<double>();
    f.nparts = std::max(1, std::min(2 * ctx->num_sms, (S.n + 255) / 256));
    return f;
}

// sum of the polynomial weights the current options use for system S (q(0))
double weight_sum(const hsc_options& o, const System& S) {
    double w = 0.0;
    if (o.preconditioner == HSC_PRECOND_LEARNED || o.preconditioner == HSC_PRECOND_BLOCK_LEARNED)
        for (int k = 0; k < kPolyOut; ++k) w += S.h_scal.wl[k];
    else if (o.preconditioner == HSC_PRECOND_POLY || o.preconditioner == HSC_PRECOND_SCHUR_POLY ||
             (o.preconditioner == HSC_PRECOND_BLOCK && o.poly_degree > 0))
        for (int k = 0; k < o.poly_degree; ++k) w += o.poly_weights[k];
    else
        w = o.neumann_order;
    return w;
}

int prepare_system(hsc_ctx* ctx, int s, const hsc_bcoo3& M, const hsc_dof_layout& L, cudaStream_t st, bool& reanalyzed) {
    if ((int)ctx->sys.size() <= s) ctx->sys.resize(s + 1);
    System& S = ctx->sys[s];
    reanalyzed = false;
    if (!same_key(S, M, L, ctx->opt)) {
        int rc = analyze(ctx, S, M, L, st);
        if (rc) return rc;
        reanalyzed = true;
    }
    return HSC_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int hsc_version(void) { return HSC_API_VERSION; }

long long hsc_kernel_launches(void) { return launch_count(); }

int hsc_debug_checks(long long* out6) {
    if (!out6) return HSC_ERR_INVALID;
    read_fail_aca(out6);
    read_fail_pcg(out6 + 2);
    read_fail_setup(out6 + 4);
    return HSC_OK;
}

int hsc_options_default(hsc_options* o) {
    if (!o) return HSC_ERR_INVALID;
    std::memset(o, 0, sizeof(*o));
    o->max_rank = 128;
    o->aca_rtol = 0.0;
    o->neumann_order = 2;
    o->omega = 0.7;
    o->max_iter = 20000;
    o->tol = 1e-6;
    o->abd_inverse = HSC_ABD_EXACT;
    o->abd_inverse_tol = 1e-5;
    o->full_residual_limit = 0.1;
    o->precision = HSC_FP64;
    o->preconditioner = HSC_PRECOND_NEUMANN;
    o->poly_degree = 0;
    o->residual_replacement = 0;
    o->refine_target = 0.0;
    o->max_refinements = 20;
    o->fallback_on_stall = 1;
    o->threads_per_row = 0;
    o->spin_limit = 20000000;
    o->check_residual = 1;
    o->trace_iterations = 0;
    o->resident = 1;
    o->fuse_update = 0;
    o->aca_cluster = 1;
    o->reorder = 1;
    o->aca_components = 1;
    o->lanczos_stats = 0;
    o->coupled_part_weight = 1.2;
    o->graph_replay = 0;
    return HSC_OK;
}

int hsc_options_reference(hsc_options* o) {
    int rc = hsc_options_default(o);
    if (rc) return rc;
    o->max_rank = 128;          // linear_hsc.cu:162-164
    o->neumann_order = 5;
    o->max_iter = 2000;
    o->abd_inverse = HSC_ABD_ADAPTIVE;
    o->omega = 0.7;
    o->tol = 1e-4;
    o->abd_inverse_tol = 1e-5;
    o->full_residual_limit = 0.1;
    return HSC_OK;
}

int hsc_create(const hsc_options* opt, hsc_ctx** out) {
    if (!out) return HSC_ERR_INVALID;
    *out = nullptr;
    hsc_options o;
    if (opt) o = *opt; else hsc_options_default(&o);
    std::string why;
    if (!validate_options(&o, why)) return HSC_ERR_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HSC_ERR_CUDA;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return HSC_ERR_CUDA;
    hsc_ctx* c = new hsc_ctx();
    c->opt = o;
    c->device = dev;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    *out = c;
    return HSC_OK;
}

void hsc_destroy(hsc_ctx* ctx) {
    if (!ctx) return;
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->ev_blk) cudaEventDestroy(ctx->ev_blk);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->ev_aca) cudaEventDestroy(ctx->ev_aca);
    if (ctx->ev_pre) cudaEventDestroy(ctx->ev_pre);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    delete ctx;
}

int hsc_set_options(hsc_ctx* ctx, const hsc_options* opt) {
    if (!ctx || !opt) return HSC_ERR_INVALID;
    std::string why;
    if (!validate_options(opt, why)) return fail(ctx, HSC_ERR_INVALID, why);
    const bool relayout = opt->precision != ctx->opt.precision || opt->max_rank != ctx->opt.max_rank ||
                          opt->threads_per_row != ctx->opt.threads_per_row;
    ctx->opt = *opt;
    if (relayout)
        for (auto& S : ctx->sys) S.analyzed = false;
    ctx->part_key_gen = -1;  // descriptors carry option values (ACA rtol, ...)
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    return HSC_OK;
}

const char* hsc_last_error(const hsc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

static int solve_impl(hsc_ctx* ctx, int count, const hsc_bcoo3* A, const hsc_dof_layout* lay,
                      const double* const* d_b, double* const* d_x, int use_graph, cudaStream_t st,
                      hsc_stats* out, int depth) {
    const hsc_options& o = ctx->opt;
    ctx->err.clear();
    int rc = ensure_common(ctx, st);
    if (rc) return rc;
    bool any_new = false;
    if ((int)ctx->sys.size() < count) ctx->sys.resize(count);  // moves only; before any analysis of this call
    std::vector<int> idx(count);
    if (depth == 0) ctx->analysis_ms = 0.0;
    const auto t_an = std::chrono::steady_clock::now();
    if (depth == 0 && ctx->pattern_volatile > 0) {
        bool changed = false;
        for (int s = 0; s < count && s < (int)ctx->sys.size(); ++s) {
            System& S = ctx->sys[s];
            if (!same_key(S, A[s], lay[s], o)) continue;  // analysed again below anyway
            unsigned long long h = 0;
            launch_pattern_hash(A[s].d_rows, A[s].d_cols, A[s].nnzb, &S.scal.as<DevScal>()->hash, st);
            CK(cudaMemcpyAsync(&h, &S.scal.as<DevScal>()->hash, sizeof(h), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (h != S.hash) { S.analyzed = false; changed = true; }
        }
        ctx->pattern_volatile = changed ? 16 : ctx->pattern_volatile - 1;
    }
    auto add_analysis_time = [&](std::chrono::steady_clock::time_point t0) {
        ctx->analysis_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    for (int s = 0; s < count; ++s) {
        bool re = false;
        rc = prepare_system(ctx, s, A[s], lay[s], st, re);
        if (rc) { if (out) out[s].status = rc; return rc; }
        any_new |= re;
        idx[s] = s;
    }
    const bool block = o.preconditioner == HSC_PRECOND_BLOCK || o.preconditioner == HSC_PRECOND_BLOCK_LEARNED;
    if (block && count != 1) return fail(ctx, HSC_ERR_INVALID, "the block preconditioner solves one system per call");
    if (any_new || ctx->part_key_gen != 2 * count + (block ? 1 : 0)) {
        ctx->block_layout = block;
        rc = build_partition(ctx, idx, st);
        if (rc) return rc;
        ctx->part_key_gen = 2 * count + (block ? 1 : 0);
        if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
        if (block) {
            rc = build_block_plan(ctx, ctx->sys[0], st);
            if (rc) return rc;
        }
        add_analysis_time(t_an);
    } else if (any_new) {
        add_analysis_time(t_an);
    }
    const bool refine = o.refine_target > 0 && count == 1;
    const bool residual = o.check_residual || refine;
    const bool learned = o.preconditioner == HSC_PRECOND_LEARNED || o.preconditioner == HSC_PRECOND_BLOCK_LEARNED;
    if (learned && !ctx->has_model) return fail(ctx, HSC_ERR_INVALID, "a learned preconditioner without a model (hsc_set_learned_model)");
    // the features of this solve see the record of the previous solve of the same system
    for (int s = 0; s < count; ++s) {
        System& S = ctx->sys[s];
        if (S.h_last[0] > 0.5) std::memcpy(S.h_prevrec, S.h_last, sizeof S.h_prevrec);
        CK(cudaMemcpyAsync(S.scal.as<DevScal>()->prev, S.h_prevrec, sizeof S.h_prevrec, cudaMemcpyHostToDevice, st));
    }
    // graph key: every pointer the numeric phase touches
    std::vector<const void*> key;
    for (int s = 0; s < count; ++s) {
        key.push_back(A[s].d_rows); key.push_back(A[s].d_cols); key.push_back(A[s].d_values);
        key.push_back(d_b[s]); key.push_back(d_x[s]);
    }
    key.push_back((const void*)st);
    const bool graph_ok = use_graph && !refine && o.abd_inverse != HSC_ABD_ADAPTIVE;
    if (use_graph && !st) return fail(ctx, HSC_ERR_INVALID, "graph replay needs a non-default stream");
    ctx->stage_events = !graph_ok && count == 1;
    CK(cudaEventRecord(ctx->ev[0], st));
    auto enqueue = [&](bool allow_sync) -> int {
        for (int s = 0; s < count; ++s) {
            int r2 = numeric_pre(ctx, ctx->sys[s], A[s], st);
            if (r2) return r2;
        }
        stage_mark(ctx, 1, st);
        // the ABD inverses (A only) run on the side stream beside the ACA (E only)
        CK(cudaEventRecord(ctx->ev_fork, st));
        CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
        for (int s = 0; s < count; ++s) {
            int r2 = abd_inverse(ctx, ctx->sys[s], ctx->side, allow_sync);
            if (r2) return r2;
        }
        CK(cudaEventRecord(ctx->ev_join, ctx->side));
        int r1 = aca_all(ctx, count, st);
        if (r1) return r1;
        stage_mark(ctx, 2, st);
        // Y = L V and G need only the ACA (and, for the learned weights, the features): side stream,
        // beside the reduced core and the rhs
        const bool pre_side = block && o.preconditioner == HSC_PRECOND_BLOCK;
        if (pre_side) {
            CK(cudaEventRecord(ctx->ev_aca, st));
            CK(cudaStreamWaitEvent(ctx->side, ctx->ev_aca, 0));
            int rb = launch_block_pre(ctx, ctx->sys[0], ctx->side);
            if (rb) return rb;
            CK(cudaEventRecord(ctx->ev_pre, ctx->side));
        }
        CK(cudaStreamWaitEvent(st, ctx->ev_join, 0));
        stage_mark(ctx, 3, st);
        for (int s = 0; s < count; ++s) {
            int r2 = numeric_post(ctx, ctx->sys[s], st);
            if (r2) return r2;
            schur_rhs(ctx->sys[s], d_b[s], st);
        }
        if (learned)
            for (int s = 0; s < count; ++s) CK(launch_features(feat_args(ctx, ctx->sys[s], true), st));
        CK(cudaEventRecord(ctx->ev[5], st));
        if (pre_side) {
            CK(cudaStreamWaitEvent(st, ctx->ev_pre, 0));
        } else if (block) {
            int rb = launch_block_pre(ctx, ctx->sys[0], st);
            if (rb) return rb;
        }
        int r3 = block ? launch_block_solve(ctx, ctx->sys[0], st) : launch_pcg_all(ctx, count, st);
        if (r3) return r3;
        CK(cudaEventRecord(ctx->ev[6], st));
        for (int s = 0; s < count; ++s) {
            back_substitute(ctx->sys[s], d_b[s], d_x[s], residual, st);
            if (residual) residual_dots(ctx, ctx->sys[s], st);
        }
        CK(cudaEventRecord(ctx->ev[7], st));
        return HSC_OK;
    };
    if (graph_ok) {
        if (!ctx->gexec || ctx->gkey != key) {
            if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            int r2 = enqueue(false);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (r2) { if (g) cudaGraphDestroy(g); return r2; }
            if (ce != cudaSuccess) return fail(ctx, HSC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&ctx->gexec, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return fail(ctx, HSC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
            ctx->gkey = key;
        }
        CK(cudaGraphLaunch(ctx->gexec, st));
    } else {
        rc = enqueue(true);
        if (rc) return rc;
    }
    CK(cudaEventRecord(ctx->ev[8], st));
    int grid_abort = 0;
    rc = read_scalars(ctx, idx, st, grid_abort);
    if (rc) return rc;
    // a pattern changed behind the same pointers: analyse again and redo once
    bool stale = false;
    for (int s = 0; s < count; ++s) stale |= ctx->sys[s].h_scal.hash != ctx->sys[s].hash;
    if (stale) {
        if (depth > 0) return fail(ctx, HSC_ERR_INVALID, "sparsity pattern changed during the solve");
        for (int s = 0; s < count; ++s) ctx->sys[s].analyzed = false;
        ctx->pattern_volatile = 16;
        return solve_impl(ctx, count, A, lay, d_b, d_x, use_graph, st, out, depth + 1);
    }
    float ms_setup = 0, ms_pcg = 0, ms_total = 0;
    float ms_stage[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (!graph_ok) {
        cudaEventElapsedTime(&ms_setup, ctx->ev[0], ctx->ev[5]);
        cudaEventElapsedTime(&ms_pcg, ctx->ev[5], ctx->ev[6]);
        cudaEventElapsedTime(&ms_stage[6], ctx->ev[6], ctx->ev[7]);
        if (ctx->stage_events)
            for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms_stage[i], ctx->ev[i], ctx->ev[i + 1]);
        ms_stage[5] = ms_pcg;
        if (block && ctx->stage_events) {  // the block form's Y / K setup, apart from the PCG proper
            cudaEventElapsedTime(&ms_stage[7], ctx->ev[5], ctx->ev_blk);
            ms_stage[5] = ms_pcg - ms_stage[7];
        }
    }
    cudaEventElapsedTime(&ms_total, ctx->ev[0], ctx->ev[8]);
    int total_iters = -1, steps = 1;
    int worst = HSC_OK;
    if (refine) {
        // quadratic refinement with exact line search (core.py:171-198):
        // x <- x + alpha d,  d = HSC(b - H x),  alpha = min(1, r.d / d.H d)
        System& S = ctx->sys[0];
        const int N = 3 * S.nblock;
        std::string msg;
        int st0 = system_status(ctx, S, S.h_scal, false, grid_abort, msg);
        if (st0) { if (out) { fill_stats(ctx, S, S.h_scal, out, false, 0, -1); out->status = st0; } return fail(ctx, st0, msg); }
        double* xacc = S.dvec[0].as<double>();
        double* res = S.dvec[1].as<double>();
        double* Hd = S.dvec[2].as<double>();
        total_iters = (int)S.h_scal.pcg[0];
        // first direction d = d_x[0] (already computed); line step from x = 0
        CK(cudaMemsetAsync(xacc, 0, sizeof(double) * N, st));
        CK(cudaMemcpyAsync(res, d_b[0], sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        double bn = 0;
        {
            launch_dot2(d_b[0], d_b[0], d_b[0], N, S.scal.as<DevScal>()->nd, st);
            double nd[2];
            CK(cudaMemcpyAsync(nd, S.scal.as<DevScal>()->nd, sizeof nd, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            bn = std::sqrt(nd[0]);
        }
        double full = 1.0;
        steps = 0;
        for (;;) {
            ++steps;
            full_spmv_contig(S, d_x[0], Hd, st);
            launch_dot2(res, d_x[0], Hd, N, S.scal.as<DevScal>()->nd, st);
            launch_line_step(xacc, d_x[0], N, S.scal.as<DevScal>()->nd, st);
            full_spmv_contig(S, xacc, Hd, st);
            launch_sub(d_b[0], Hd, res, N, st);
            launch_dot2(res, res, res, N, S.scal.as<DevScal>()->resid, st);
            double h2[2];
            CK(cudaMemcpyAsync(h2, S.scal.as<DevScal>()->resid, sizeof h2, cudaMemcpyDeviceToHost, st));
            double nd[2];
            CK(cudaMemcpyAsync(nd, S.scal.as<DevScal>()->nd, sizeof nd, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (!(nd[0] > 0 && nd[1] > 0)) {
                worst = HSC_ERR_NONDESCENT;
                ctx->err = "approximate HSC direction is not descent";
                break;
            }
            full = bn > 0 ? std::sqrt(h2[0]) / bn : 0.0;
            if (full <= o.refine_target || steps >= o.max_refinements) break;
            // next direction
            schur_rhs(S, res, st);
            int r4 = block ? launch_block_solve(ctx, S, st) : launch_pcg_all(ctx, 1, st);
            if (r4) return r4;
            back_substitute(S, res, d_x[0], false, st);
            int ga = 0;
            r4 = read_scalars(ctx, idx, st, ga);
            if (r4) return r4;
            total_iters += (int)S.h_scal.pcg[0];
            st0 = system_status(ctx, S, S.h_scal, false, ga, msg);
            if (st0) { worst = st0; ctx->err = msg; break; }
        }
        CK(cudaMemcpyAsync(d_x[0], xacc, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
        // final full residual and descent with the accumulated x
        launch_dot2(d_b[0], d_x[0], d_x[0], N, S.scal.as<DevScal>()->nd, st);
        double nd[2];
        CK(cudaMemcpyAsync(nd, S.scal.as<DevScal>()->nd, sizeof nd, cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(ctx->ev[8], st));
        CK(cudaStreamSynchronize(st));
        cudaEventElapsedTime(&ms_total, ctx->ev[0], ctx->ev[8]);
        S.h_scal.resid[0] = full * full * bn * bn;
        S.h_scal.resid[1] = bn * bn;
        S.h_scal.resid[2] = nd[0];
        if (!worst && full > o.refine_target) {
            worst = HSC_ERR_NOCONV;
            ctx->err = "refinement did not reach refine_target";
        }
    }
    // Lanczos extremes of every system (host bisection, independent per system): a batch spreads
    // them over a few host threads
    std::vector<double> lz_lo(count, 0.0), lz_hi(count, 0.0);
    if (learned || o.lanczos_stats) {
        auto lz = [&](int s0, int s1) {
            for (int s = s0; s < s1; ++s) {
                const System& S = ctx->sys[s];
                const int m = std::min(kMaxCoef, std::max(0, (int)S.h_scal.pcg[0]));
                lanczos_extremes(S.h_cg, m, lz_lo[s], lz_hi[s]);
            }
        };
        const int nth = count >= 8 ? std::min(8, (int)std::max(1u, std::thread::hardware_concurrency())) : 1;
        if (nth <= 1) {
            lz(0, count);
        } else {
            std::vector<std::thread> pool;
            for (int t = 1; t < nth; ++t) pool.emplace_back(lz, count * t / nth, count * (t + 1) / nth);
            lz(0, count / nth);
            for (auto& th : pool) th.join();
        }
    }
    for (int s = 0; s < count; ++s) {
        System& S = ctx->sys[s];
        std::string msg;
        int st_s = system_status(ctx, S, S.h_scal, residual, grid_abort, msg);
        if (refine && worst) st_s = worst;
        if (out) {
            fill_stats(ctx, S, S.h_scal, out + s, residual, refine ? steps : 1, refine ? total_iters : -1);
            out[s].status = st_s;
            out[s].setup_ms = ms_setup;
            out[s].pcg_ms = ms_pcg;
            out[s].total_ms = ms_total;
            out[s].analysis_ms = ctx->analysis_ms;
            for (int i = 0; i < 8; ++i) out[s].stage_ms[i] = ms_stage[i];
            out[s].accepted = st_s == HSC_OK;
            out[s].fallback = 0;
        }
        // Lanczos extremes of this solve; they become the next solve's record
        const int m = std::min(kMaxCoef, std::max(0, (int)S.h_scal.pcg[0]));
        const double lo = lz_lo[s], hi = lz_hi[s];
        if (out) { out[s].lanczos_min = lo; out[s].lanczos_max = hi; }
        if (m > 0 && lo > 0) {
            S.h_last[0] = 1.0; S.h_last[1] = lo; S.h_last[2] = hi; S.h_last[3] = S.h_scal.pcg[0];
            S.h_last[4] = weight_sum(o, S);
        }
        if (st_s && !worst) { worst = st_s; ctx->err = msg; }
    }
    // a stalled polynomial / learned preconditioner: redo with the plain Neumann series
    if (count == 1 && !refine && depth == 0 && o.fallback_on_stall && o.preconditioner != HSC_PRECOND_NEUMANN &&
        (worst == HSC_ERR_BREAKDOWN || worst == HSC_ERR_NOCONV)) {
        const hsc_options saved = ctx->opt;
        ctx->opt.preconditioner = HSC_PRECOND_NEUMANN;
        ctx->part_key_gen = -1;
        const int iters_first = out ? out[0].pcg_iterations : 0;
        const int r = solve_impl(ctx, count, A, lay, d_b, d_x, use_graph, st, out, depth + 1);
        ctx->opt = saved;
        ctx->part_key_gen = -1;
        if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
        if (out) { out[0].fallback = 1; out[0].pcg_iterations += iters_first; }
        return r;
    }
    // in a batch, the stalled systems alone are solved again with the plain Neumann series (one
    // sub-batch, direct launches; their stats replace theirs, the iterations add up)
    if (count > 1 && out && !refine && depth == 0 && o.fallback_on_stall && o.preconditioner != HSC_PRECOND_NEUMANN &&
        o.preconditioner != HSC_PRECOND_BLOCK && o.preconditioner != HSC_PRECOND_BLOCK_LEARNED) {
        std::vector<int> bad;
        for (int s = 0; s < count; ++s)
            if (out[s].status == HSC_ERR_BREAKDOWN || out[s].status == HSC_ERR_NOCONV) bad.push_back(s);
        if (!bad.empty()) {
            const int nb = (int)bad.size();
            std::vector<hsc_bcoo3> Ab(nb);
            std::vector<hsc_dof_layout> Lb(nb);
            std::vector<const double*> bb(nb);
            std::vector<double*> xb(nb);
            std::vector<hsc_stats> ob(nb);
            for (int i = 0; i < nb; ++i) { Ab[i] = A[bad[i]]; Lb[i] = lay[bad[i]]; bb[i] = d_b[bad[i]]; xb[i] = d_x[bad[i]]; }
            const hsc_options saved = ctx->opt;
            ctx->opt.preconditioner = HSC_PRECOND_NEUMANN;
            ctx->part_key_gen = -1;
            if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
            solve_impl(ctx, nb, Ab.data(), Lb.data(), bb.data(), xb.data(), 0, st, ob.data(), depth + 1);
            ctx->opt = saved;
            ctx->part_key_gen = -1;
            if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
            for (int i = 0; i < nb; ++i) {
                const int iters_first = out[bad[i]].pcg_iterations;
                out[bad[i]] = ob[i];
                out[bad[i]].fallback = 1;
                out[bad[i]].pcg_iterations += iters_first;
            }
            worst = HSC_OK;
            for (int s = 0; s < count; ++s)
                if (out[s].status && !worst) worst = out[s].status;
        }
    }
    return worst;
}

int hsc_solve(hsc_ctx* ctx, const hsc_bcoo3* A, const hsc_dof_layout* layout, const double* d_b, double* d_x,
              void* stream, hsc_stats* out) {
    if (!ctx || !A || !layout || !d_b || !d_x) return HSC_ERR_INVALID;
    const int graph = ctx->opt.graph_replay && stream != nullptr ? 1 : 0;
    int rc = solve_impl(ctx, 1, A, layout, &d_b, &d_x, graph, (cudaStream_t)stream, out, 0);
    if (rc && out && out->status == 0) out->status = rc;
    return rc;
}

int hsc_solve_batch(hsc_ctx* ctx, int32_t count, const hsc_bcoo3* A, const hsc_dof_layout* layouts,
                    const double* const* d_b, double* const* d_x, int32_t use_graph, void* stream, hsc_stats* out) {
    if (!ctx || count < 1 || !A || !layouts || !d_b || !d_x) return HSC_ERR_INVALID;
    return solve_impl(ctx, count, A, layouts, d_b, d_x, use_graph, (cudaStream_t)stream, out, 0);
}

int hsc_spmv(hsc_ctx* ctx, const hsc_bcoo3* A, const hsc_dof_layout* layout, const double* d_x, double* d_y,
             void* stream) {
    if (!ctx || !A || !layout || !d_x || !d_y) return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->err.clear();
    int rc = ensure_common(ctx, st);
    if (rc) return rc;
    bool re = false;
    rc = prepare_system(ctx, 0, *A, *layout, st, re);
    if (rc) return rc;
    System& S = ctx->sys[0];
    DevScal* ds = S.scal.as<DevScal>();
    launch_extract(S.qq.as<int>(), S.nqq, S.qf.as<int>(), S.nqf, A->d_values, S.qm, S.a, S.A.as<double>(),
                   S.E.as<double>(), S.node_nz.as<int>(), st);
    (void)ds;
    full_spmv_contig(S, d_x, d_y, st, A->d_values);  // FEM blocks straight from the BCOO: no BSR refill
    CK(cudaStreamSynchronize(st));
    if (re) ctx->part_key_gen = -1;
    return HSC_OK;
}

int hsc_get_factors(hsc_ctx* ctx, int32_t sys, int32_t* rank, int32_t* n_active, double* U, int32_t ldu, double* V,
                    int32_t ldv, int32_t* active) {
    if (!ctx || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed) return HSC_ERR_NOTREADY;
    System& S = ctx->sys[sys];
    const int k = S.h_scal.rank;
    if (rank) *rank = k;
    if (n_active) *n_active = S.a;
    if (active && S.a) std::memcpy(active, S.h_act.data(), sizeof(int) * S.a);
    if (U && k) CK(cudaMemcpy2D(U, sizeof(double) * ldu, S.U.p, sizeof(double) * S.qm, sizeof(double) * S.qm, k,
                                 cudaMemcpyDeviceToHost));
    if (V && k) CK(cudaMemcpy2D(V, sizeof(double) * ldv, S.V.p, sizeof(double) * S.a, sizeof(double) * S.a, k,
                                 cudaMemcpyDeviceToHost));
    return HSC_OK;
}

int hsc_get_trace(hsc_ctx* ctx, unsigned long long* out, int64_t max_entries, int32_t* ctas, int32_t* iterations) {
    if (!ctx || ctx->opt.trace_iterations <= 0 || !ctx->d_trace.p) return HSC_ERR_NOTREADY;
    const int64_t nt = (int64_t)ctx->grid * ctx->opt.trace_iterations * kTraceEvents;
    if (ctas) *ctas = ctx->grid;
    if (iterations) *iterations = ctx->opt.trace_iterations;
    if (out) CK(cudaMemcpy(out, ctx->d_trace.p, sizeof(unsigned long long) * std::min(nt, max_entries),
                           cudaMemcpyDeviceToHost));
    return HSC_OK;
}

int hsc_set_learned_model(hsc_ctx* ctx, const uint16_t* params_bf16) {
    if (!ctx || !params_bf16) return HSC_ERR_INVALID;
    GROW(ctx->mlp, sizeof(uint16_t) * kParams);
    CK(cudaMemcpy(ctx->mlp.p, params_bf16, sizeof(uint16_t) * kParams, cudaMemcpyHostToDevice));
    ctx->has_model = true;
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    return HSC_OK;
}

int hsc_get_features(hsc_ctx* ctx, int32_t sys, float* out) {
    if (!ctx || !out || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed) return HSC_ERR_NOTREADY;
    System& S = ctx->sys[sys];
    int rc = ensure_common(ctx, nullptr);
    if (rc) return rc;
    CK(launch_features(feat_args(ctx, S, false), nullptr));
    CK(cudaMemcpy(out, S.scal.as<DevScal>()->feat, sizeof(float) * kFeat, cudaMemcpyDeviceToHost));
    return HSC_OK;
}

int hsc_get_poly_weights(hsc_ctx* ctx, int32_t sys, double* out, int32_t max, int32_t* degree) {
    if (!ctx || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed) return HSC_ERR_NOTREADY;
    const hsc_options& o = ctx->opt;
    const System& S = ctx->sys[sys];
    std::vector<double> w;
    if (o.preconditioner == HSC_PRECOND_LEARNED) w.assign(S.h_scal.wl, S.h_scal.wl + kPolyOut);
    else if (o.preconditioner == HSC_PRECOND_POLY || o.preconditioner == HSC_PRECOND_SCHUR_POLY)
        w.assign(o.poly_weights, o.poly_weights + o.poly_degree);
    else w.assign(o.neumann_order, 1.0);
    if (degree) *degree = (int)w.size();
    if (out)
        for (int k = 0; k < std::min<int>(max, (int)w.size()); ++k) out[k] = w[k];
    return HSC_OK;
}

int hsc_get_lanczos(hsc_ctx* ctx, int32_t sys, double* coef, int32_t max_pairs, int32_t* pairs) {
    if (!ctx || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed) return HSC_ERR_NOTREADY;
    const System& S = ctx->sys[sys];
    const int m = std::min(kMaxCoef, std::max(0, (int)S.h_scal.pcg[0]));
    const int k = std::min<int>(m, std::max(0, max_pairs));
    if (pairs) *pairs = k;
    if (coef) std::memcpy(coef, S.h_cg, sizeof(double) * 2 * k);
    return HSC_OK;
}

int hsc_get_partition(hsc_ctx* ctx, int32_t sys, int32_t* n, int32_t* nparts, int32_t* perm, int32_t* part_ptr) {
    if (!ctx || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed) return HSC_ERR_NOTREADY;
    const System& S = ctx->sys[sys];
    if (n) *n = S.n;
    if (nparts) *nparts = (int)S.h_part_ptr.size() - 1;
    if (perm && S.n) std::memcpy(perm, S.h_perm.data(), sizeof(int) * S.n);
    if (part_ptr) std::memcpy(part_ptr, S.h_part_ptr.data(), sizeof(int) * S.h_part_ptr.size());
    return HSC_OK;
}

int hsc_debug_block_plan(hsc_ctx* ctx, int64_t* out, int32_t n) {
    if (!ctx || !out || n < 1) return HSC_ERR_INVALID;
    if (ctx->sys.empty() || !ctx->block_layout) return HSC_ERR_NOTREADY;
    const BlockPlan& b = ctx->sys[0].blk;
    const int64_t v[] = {b.G_ctas, b.R, b.NS, b.NCH, b.W, b.NA, b.NCOL, b.stage_vals, b.NYC,
                         (int64_t)b.smem, (int64_t)b.smem_y, b.ncomp, b.nslot, b.kmax};
    for (int i = 0; i < n && i < (int)(sizeof v / sizeof v[0]); ++i) out[i] = v[i];
    return HSC_OK;
}

int hsc_partition_nodes(int32_t n, const int32_t* adj_ptr, const int32_t* adj, const double* weight, int32_t nparts,
                        int32_t* part) {
    if (n < 0 || nparts < 1 || (n > 0 && (!adj_ptr || !adj || !weight || !part))) return HSC_ERR_INVALID;
    if (n == 0) return HSC_OK;
    std::vector<int> ptr(adj_ptr, adj_ptr + n + 1);
    if (ptr[0] != 0) return HSC_ERR_INVALID;
    for (int i = 0; i < n; ++i)
        if (ptr[i + 1] < ptr[i] || !(weight[i] > 0)) return HSC_ERR_INVALID;
    std::vector<int> a(adj, adj + ptr[n]);
    for (int v : a)
        if (v < 0 || v >= n) return HSC_ERR_INVALID;
    std::vector<double> w(weight, weight + n);
    const std::vector<int> p = partition_nodes(n, ptr, a, w, nparts);
    std::memcpy(part, p.data(), sizeof(int) * n);
    return HSC_OK;
}

int hsc_get_abd_inverse(hsc_ctx* ctx, int32_t sys, double* P) {
    if (!ctx || sys < 0 || sys >= (int)ctx->sys.size() || !ctx->sys[sys].analyzed || !P) return HSC_ERR_NOTREADY;
    System& S = ctx->sys[sys];
    if (S.qm) CK(cudaMemcpy(P, S.P.p, sizeof(double) * S.qm * S.qm, cudaMemcpyDeviceToHost));
    return HSC_OK;
}

}  // extern "C"
