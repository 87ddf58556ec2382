// GPU assembly of the ABD-FEM contact coupling, fused with the extraction of
// the HSC solver's active FEM columns and of its ACA input E.
//
// Per contact (reference: ABDFEMLinearSubsystem_assemble_kernel,
// abd_fem_linear_subsystem.cu:18-61): the 3x3 Hessian block H between an
// affine-body vertex (rest position xbar) and a FEM node is pulled back to
// the body's 12 dofs, H12x3 = J(xbar)^T H, and zeroed when the body or the
// FEM node is fixed; it becomes the four 3x3 blocks (4 body + k, node) of the
// global matrix's upper triangle (ABD dofs come before FEM dofs).
// J(xbar) is the 3x12 affine map q -> x: x = p + [a1.xbar, a2.xbar, a3.xbar]
// with q = (p, a1, a2, a3) (p_first = 1, libuipc's ABD order) or
// q = (a1, a2, a3, p) (p_first = 0, the order of the reference's NumPy core).
//
// The same pass produces what the solver's setup would otherwise rebuild on
// the host from the assembled matrix (linear_hsc.cu:205-247): the sorted FEM
// dofs of the nodes with a coupling block of nonzero squared norm and the
// dense E (qm x a, row-major) over them, the ACA input.
//
// Determinism: contacts are stably radix-sorted by (body, node); each
// (body, node) pair sums its contacts in input order; output positions come
// from prefix sums -- no floating-point atomics, bit-identical repeats.
#include <algorithm>
#include <cstdint>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "../../include/hsc_c_api.h"
#include "hsc_internal.cuh"

namespace hsc {
namespace {

constexpr int kT = 256;
inline int nblocks_for(long long n) { return (int)std::max<long long>(1, (n + kT - 1) / kT); }

struct Counters {
    int npairs, nkept, nact, bad;
};

__global__ void keys_kernel(const int* __restrict__ abd_v, const int* __restrict__ fem_v, int n,
                            const int* __restrict__ v2b, int nabd_v, int nbody, int nfem,
                            unsigned long long* __restrict__ keys, int* __restrict__ idx, Counters* cnt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int v = abd_v[t], f = fem_v[t];
    unsigned long long key = (unsigned long long)nbody << 32;  // invalid: sorts after every body
    if (v >= 0 && v < nabd_v && f >= 0 && f < nfem) {
        const int b = v2b[v];
        if (b >= 0 && b < nbody) key = ((unsigned long long)b << 32) | (unsigned)f;
        else atomicAdd(&cnt->bad, 1);
    } else {
        atomicAdd(&cnt->bad, 1);
    }
    keys[t] = key;
    idx[t] = t;
}

__global__ void head_kernel(const unsigned long long* __restrict__ keys, int n, int nbody, int* __restrict__ head) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool valid = (keys[i] >> 32) < (unsigned long long)nbody;
    head[i] = valid && (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void pair_start_kernel(const int* __restrict__ head, const int* __restrict__ pid, int n,
                                  int* __restrict__ pstart, Counters* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (head[i]) pstart[pid[i]] = i;
    if (i == n - 1) cnt->npairs = pid[i] + head[i];
}

// (J^T H)[c][j] for one contact block H (column-major, H(r, j) at r + 3 j); each entry is one rounded
// product, added to the pair's sum as its own rounded term (no fused multiply-add), as a sum of
// assembled triplets rounds it
__device__ __forceinline__ double jth(const double* H, const double* xb, int c, int j, int p_first) {
    if (p_first) {
        if (c < 3) return H[c + 3 * j];
        const int r = (c - 3) / 3, m = (c - 3) % 3;
        return __dmul_rn(xb[m], H[r + 3 * j]);
    }
    if (c >= 9) return H[(c - 9) + 3 * j];
    return __dmul_rn(xb[c % 3], H[c / 3 + 3 * j]);
}

// one thread per (body, node) pair: the 12x3 sum of its contacts in input order
__global__ void pair_sum_kernel(const unsigned long long* __restrict__ keys, const int* __restrict__ idx, int n,
                                const int* __restrict__ pstart, const int* __restrict__ abd_v,
                                const double* __restrict__ xbar, const double* __restrict__ H,
                                const int* __restrict__ body_fixed, const int* __restrict__ fem_fixed, int p_first,
                                const Counters* cnt, double* __restrict__ pairbuf, int* __restrict__ keep,
                                int* __restrict__ blocknz) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (p >= cnt->npairs) { keep[p] = 0; return; }
    const int i0 = pstart[p];
    const unsigned long long key = keys[i0];
    const int b = (int)(key >> 32), f = (int)(key & 0xffffffffu);
    double acc[36];
    for (int e = 0; e < 36; ++e) acc[e] = 0.0;
    const bool fixed = (body_fixed && body_fixed[b]) || (fem_fixed && fem_fixed[f]);
    if (!fixed) {
        for (int i = i0; i < n && keys[i] == key; ++i) {
            const int t = idx[i];
            const double* Ht = H + 9 * (size_t)t;
            const double* xb = xbar + 3 * (size_t)abd_v[t];
            for (int c = 0; c < 12; ++c)
                for (int j = 0; j < 3; ++j) acc[3 * c + j] = __dadd_rn(acc[3 * c + j], jth(Ht, xb, c, j, p_first));
        }
    }
    int nzmask = 0;
    for (int k = 0; k < 4; ++k) {
        double sq = 0.0;
        for (int e = 0; e < 9; ++e) sq += acc[9 * k + e] * acc[9 * k + e];
        if (sq != 0.0) nzmask |= 1 << k;
    }
    double* out = pairbuf + 36 * (size_t)p;
    for (int e = 0; e < 36; ++e) out[e] = acc[e];
    keep[p] = nzmask != 0;
    blocknz[p] = nzmask;
}

__global__ void compact_kernel(const int* __restrict__ keep, const int* __restrict__ kpos, int n,
                               int* __restrict__ kept, Counters* cnt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (keep[p]) kept[kpos[p]] = p;
    if (p == n - 1) cnt->nkept = kpos[p] + keep[p];
}

__global__ void body_range_kernel(const int* __restrict__ kept, const unsigned long long* __restrict__ keys,
                                  const int* __restrict__ pstart, int n, const Counters* cnt,
                                  int* __restrict__ bfirst, int* __restrict__ blast, int* __restrict__ node_flag) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nk = cnt->nkept;
    if (q >= n || q >= nk) return;
    const unsigned long long key = keys[pstart[kept[q]]];
    const int b = (int)(key >> 32);
    if (q == 0 || (int)(keys[pstart[kept[q - 1]]] >> 32) != b) bfirst[b] = q;
    if (q == nk - 1 || (int)(keys[pstart[kept[q + 1]]] >> 32) != b) blast[b] = q;
    node_flag[key & 0xffffffffu] = 1;
}

// the four upper-triangle blocks of each kept pair, sorted by (row, col)
__global__ void write_blocks_kernel(const int* __restrict__ kept, const unsigned long long* __restrict__ keys,
                                    const int* __restrict__ pstart, const double* __restrict__ pairbuf, int n,
                                    const Counters* cnt, const int* __restrict__ bfirst, const int* __restrict__ blast,
                                    int abd_off, int fem_off, int* __restrict__ rows, int* __restrict__ cols,
                                    double* __restrict__ vals) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n || q >= cnt->nkept) return;
    const int p = kept[q];
    const unsigned long long key = keys[pstart[p]];
    const int b = (int)(key >> 32), f = (int)(key & 0xffffffffu);
    const int bs = bfirst[b], nb = blast[b] - bs + 1;
    const double* src = pairbuf + 36 * (size_t)p;
    for (int k = 0; k < 4; ++k) {
        const size_t o = 4 * (size_t)bs + (size_t)k * nb + (q - bs);
        rows[o] = abd_off + 4 * b + k;
        cols[o] = fem_off + f;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) vals[9 * o + i + 3 * j] = src[3 * (3 * k + i) + j];
    }
}

__global__ void active_kernel(const int* __restrict__ node_flag, const int* __restrict__ node_pos, int nfem,
                              int fem_dof_off, int* __restrict__ act, Counters* cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfem) return;
    if (node_flag[i])
        for (int j = 0; j < 3; ++j) act[3 * node_pos[i] + j] = fem_dof_off + 3 * i + j;
    if (i == nfem - 1) cnt->nact = node_pos[i] + node_flag[i];
}

// E (qm x a, row-major): block k of a kept pair where its squared norm is nonzero
__global__ void fill_E_kernel(const int* __restrict__ kept, const unsigned long long* __restrict__ keys,
                              const int* __restrict__ pstart, const double* __restrict__ pairbuf,
                              const int* __restrict__ blocknz, const int* __restrict__ node_pos, int nkept, int a,
                              double* __restrict__ E) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nkept) return;
    const int p = kept[q];
    const unsigned long long key = keys[pstart[p]];
    const int b = (int)(key >> 32), f = (int)(key & 0xffffffffu);
    const int c = node_pos[f], nz = blocknz[p];
    const double* src = pairbuf + 36 * (size_t)p;
    for (int k = 0; k < 4; ++k) {
        if (!(nz >> k & 1)) continue;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) E[(size_t)(12 * b + 3 * k + i) * a + 3 * c + j] = src[3 * (3 * k + i) + j];
    }
}

}  // namespace
}  // namespace hsc

struct hsc_coupling_assembler {
    int nabd_v = 0, nbody = 0, nfem = 0, abd_off = 0, fem_off = 0, p_first = 1;
    int* v2b = nullptr;          // device nabd_v
    double* xbar = nullptr;      // device nabd_v x 3
    int* body_fixed = nullptr;   // device nbody, or null
    int* fem_fixed = nullptr;    // device nfem, or null
    hsc::Counters* cnt = nullptr;
    // per-call buffers, grown on demand
    int cap = 0;
    unsigned long long *keys_in = nullptr, *keys = nullptr;
    int *idx_in = nullptr, *idx = nullptr, *head = nullptr, *pid = nullptr, *pstart = nullptr;
    int *keep = nullptr, *kpos = nullptr, *kept = nullptr, *blocknz = nullptr;
    double* pairbuf = nullptr;
    int *rows = nullptr, *cols = nullptr;
    double* vals = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    int *bfirst = nullptr, *blast = nullptr, *node_flag = nullptr, *node_pos = nullptr, *act = nullptr;
    double* E = nullptr;
    size_t E_cap = 0;
    int nkept = 0, nact = 0;
};

namespace {
void free_per_call(hsc_coupling_assembler* a) {
    cudaFree(a->keys_in); cudaFree(a->keys); cudaFree(a->idx_in); cudaFree(a->idx); cudaFree(a->head);
    cudaFree(a->pid); cudaFree(a->pstart); cudaFree(a->keep); cudaFree(a->kpos); cudaFree(a->kept);
    cudaFree(a->blocknz); cudaFree(a->pairbuf); cudaFree(a->rows); cudaFree(a->cols); cudaFree(a->vals);
    cudaFree(a->tmp);
    a->keys_in = a->keys = nullptr;
    a->idx_in = a->idx = a->head = a->pid = a->pstart = a->keep = a->kpos = a->kept = a->blocknz = nullptr;
    a->pairbuf = nullptr; a->rows = a->cols = nullptr; a->vals = nullptr; a->tmp = nullptr;
    a->cap = 0; a->tmp_bytes = 0;
}
void free_coupling(hsc_coupling_assembler* a) {
    if (!a) return;
    free_per_call(a);
    cudaFree(a->v2b); cudaFree(a->xbar); cudaFree(a->body_fixed); cudaFree(a->fem_fixed); cudaFree(a->cnt);
    cudaFree(a->bfirst); cudaFree(a->blast); cudaFree(a->node_flag); cudaFree(a->node_pos); cudaFree(a->act);
    cudaFree(a->E);
    delete a;
}
template <class T> cudaError_t alloc_n(T** p, size_t n) { return cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(1, n)); }
template <class T> cudaError_t upload_n(T** d, const T* h, size_t n) {
    cudaError_t e = alloc_n(d, n);
    if (e == cudaSuccess && n) e = cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice);
    return e;
}
int key_bits(int nbody) {  // bits of (body << 32 | node) the sort must look at, the invalid key included
    int b = 0;
    while ((1ll << b) <= nbody) ++b;
    return 32 + b;
}
int grow(hsc_coupling_assembler* a, int n) {
    if (n <= a->cap) return HSC_OK;
    free_per_call(a);
    const int c = std::max(n, 1024);
    bool ok = alloc_n(&a->keys_in, c) == cudaSuccess && alloc_n(&a->keys, c) == cudaSuccess &&
              alloc_n(&a->idx_in, c) == cudaSuccess && alloc_n(&a->idx, c) == cudaSuccess &&
              alloc_n(&a->head, c) == cudaSuccess && alloc_n(&a->pid, c) == cudaSuccess &&
              alloc_n(&a->pstart, c) == cudaSuccess && alloc_n(&a->keep, c) == cudaSuccess &&
              alloc_n(&a->kpos, c) == cudaSuccess && alloc_n(&a->kept, c) == cudaSuccess &&
              alloc_n(&a->blocknz, c) == cudaSuccess && alloc_n(&a->pairbuf, 36 * (size_t)c) == cudaSuccess &&
              alloc_n(&a->rows, 4 * (size_t)c) == cudaSuccess && alloc_n(&a->cols, 4 * (size_t)c) == cudaSuccess &&
              alloc_n(&a->vals, 36 * (size_t)c) == cudaSuccess;
    if (!ok) { free_per_call(a); return HSC_ERR_ALLOC; }
    size_t s1 = 0, s2 = 0, s3 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, s1, a->keys_in, a->keys, a->idx_in, a->idx, c, 0, key_bits(a->nbody));
    cub::DeviceScan::ExclusiveSum(nullptr, s2, a->head, a->pid, c);
    cub::DeviceScan::ExclusiveSum(nullptr, s3, a->node_flag, a->node_pos, std::max(1, a->nfem));
    a->tmp_bytes = std::max({s1, s2, s3, (size_t)256});
    if (cudaMalloc(&a->tmp, a->tmp_bytes) != cudaSuccess) { free_per_call(a); return HSC_ERR_ALLOC; }
    a->cap = c;
    return HSC_OK;
}
}  // namespace

#define CC(x) do { if ((x) != cudaSuccess) return HSC_ERR_CUDA; } while (0)

extern "C" {

int hsc_coupling_assembler_create(int32_t n_abd_vertices, const int32_t* v2b, const double* x_bar, int32_t nbody,
                                  const int32_t* body_fixed, int32_t nfem, const int32_t* fem_fixed,
                                  int32_t abd_block_offset, int32_t fem_block_offset, int32_t p_first,
                                  hsc_coupling_assembler** out) {
    if (!out || !v2b || !x_bar || n_abd_vertices < 1 || nbody < 1 || nfem < 1 || abd_block_offset < 0 ||
        fem_block_offset < 0 || nbody >= (1 << 26))
        return HSC_ERR_INVALID;
    *out = nullptr;
    for (int v = 0; v < n_abd_vertices; ++v)
        if (v2b[v] < 0 || v2b[v] >= nbody) return HSC_ERR_INVALID;
    auto* a = new hsc_coupling_assembler();
    a->nabd_v = n_abd_vertices; a->nbody = nbody; a->nfem = nfem;
    a->abd_off = abd_block_offset; a->fem_off = fem_block_offset; a->p_first = p_first ? 1 : 0;
    bool ok = upload_n(&a->v2b, v2b, n_abd_vertices) == cudaSuccess &&
              upload_n(&a->xbar, x_bar, 3 * (size_t)n_abd_vertices) == cudaSuccess &&
              (!body_fixed || upload_n(&a->body_fixed, body_fixed, nbody) == cudaSuccess) &&
              (!fem_fixed || upload_n(&a->fem_fixed, fem_fixed, nfem) == cudaSuccess) &&
              alloc_n(&a->cnt, 1) == cudaSuccess && alloc_n(&a->bfirst, nbody) == cudaSuccess &&
              alloc_n(&a->blast, nbody) == cudaSuccess && alloc_n(&a->node_flag, nfem) == cudaSuccess &&
              alloc_n(&a->node_pos, nfem) == cudaSuccess && alloc_n(&a->act, 3 * (size_t)nfem) == cudaSuccess;
    if (!ok) { free_coupling(a); return HSC_ERR_ALLOC; }
    *out = a;
    return HSC_OK;
}

int hsc_coupling_assembler_destroy(hsc_coupling_assembler* a) {
    free_coupling(a);
    return HSC_OK;
}

int hsc_coupling_assemble(hsc_coupling_assembler* a, const int32_t* d_abd_vertex, const int32_t* d_fem_vertex,
                          const double* d_H, int32_t ncontact, int32_t* nblocks, int32_t* nactive, void* stream) {
    if (!a || ncontact < 0 || (ncontact > 0 && (!d_abd_vertex || !d_fem_vertex || !d_H)) ||
        ncontact > (1 << 28))
        return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    a->nkept = a->nact = 0;
    if (nblocks) *nblocks = 0;
    if (nactive) *nactive = 0;
    if (ncontact == 0) return HSC_OK;
    int rc = grow(a, ncontact);
    if (rc) return rc;
    const int n = ncontact, g = hsc::nblocks_for(n);
    using namespace hsc;
    CC(cudaMemsetAsync(a->cnt, 0, sizeof(Counters), st));
    CC(cudaMemsetAsync(a->node_flag, 0, sizeof(int) * a->nfem, st));
    count_launch();
    keys_kernel<<<g, kT, 0, st>>>(d_abd_vertex, d_fem_vertex, n, a->v2b, a->nabd_v, a->nbody, a->nfem, a->keys_in,
                                  a->idx_in, a->cnt);
    size_t tb = a->tmp_bytes;
    CC(cub::DeviceRadixSort::SortPairs(a->tmp, tb, a->keys_in, a->keys, a->idx_in, a->idx, n, 0,
                                       key_bits(a->nbody), st));
    count_launch();
    head_kernel<<<g, kT, 0, st>>>(a->keys, n, a->nbody, a->head);
    tb = a->tmp_bytes;
    CC(cub::DeviceScan::ExclusiveSum(a->tmp, tb, a->head, a->pid, n, st));
    count_launch();
    pair_start_kernel<<<g, kT, 0, st>>>(a->head, a->pid, n, a->pstart, a->cnt);
    count_launch();
    pair_sum_kernel<<<g, kT, 0, st>>>(a->keys, a->idx, n, a->pstart, d_abd_vertex, a->xbar, d_H, a->body_fixed,
                                      a->fem_fixed, a->p_first, a->cnt, a->pairbuf, a->keep, a->blocknz);
    tb = a->tmp_bytes;
    CC(cub::DeviceScan::ExclusiveSum(a->tmp, tb, a->keep, a->kpos, n, st));
    count_launch();
    compact_kernel<<<g, kT, 0, st>>>(a->keep, a->kpos, n, a->kept, a->cnt);
    count_launch();
    body_range_kernel<<<g, kT, 0, st>>>(a->kept, a->keys, a->pstart, n, a->cnt, a->bfirst, a->blast, a->node_flag);
    count_launch();
    write_blocks_kernel<<<g, kT, 0, st>>>(a->kept, a->keys, a->pstart, a->pairbuf, n, a->cnt, a->bfirst, a->blast,
                                          a->abd_off, a->fem_off, a->rows, a->cols, a->vals);
    tb = a->tmp_bytes;
    CC(cub::DeviceScan::ExclusiveSum(a->tmp, tb, a->node_flag, a->node_pos, a->nfem, st));
    count_launch();
    active_kernel<<<nblocks_for(a->nfem), kT, 0, st>>>(a->node_flag, a->node_pos, a->nfem, 3 * a->fem_off, a->act,
                                                       a->cnt);
    CC(cudaGetLastError());
    Counters h{};
    CC(cudaMemcpyAsync(&h, a->cnt, sizeof h, cudaMemcpyDeviceToHost, st));
    CC(cudaStreamSynchronize(st));
    if (h.bad) return HSC_ERR_INVALID;
    a->nkept = h.nkept;
    a->nact = 3 * h.nact;
    const size_t qm = 12 * (size_t)a->nbody, need = qm * (size_t)a->nact;
    if (need > a->E_cap) {
        cudaFree(a->E);
        a->E = nullptr;
        a->E_cap = 0;
        if (alloc_n(&a->E, need) != cudaSuccess) return HSC_ERR_ALLOC;
        a->E_cap = need;
    }
    if (need) {
        CC(cudaMemsetAsync(a->E, 0, sizeof(double) * need, st));
        count_launch();
        fill_E_kernel<<<nblocks_for(a->nkept), kT, 0, st>>>(a->kept, a->keys, a->pstart, a->pairbuf, a->blocknz,
                                                           a->node_pos, a->nkept, a->nact, a->E);
        CC(cudaGetLastError());
    }
    if (nblocks) *nblocks = 4 * a->nkept;
    if (nactive) *nactive = a->nact;
    return HSC_OK;
}

int hsc_coupling_read(hsc_coupling_assembler* a, int32_t* d_rows, int32_t* d_cols, double* d_values,
                      int32_t* d_active, double* d_E, void* stream) {
    if (!a) return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nb = 4 * (size_t)a->nkept;
    if (nb) {
        if (d_rows) CC(cudaMemcpyAsync(d_rows, a->rows, sizeof(int) * nb, cudaMemcpyDeviceToDevice, st));
        if (d_cols) CC(cudaMemcpyAsync(d_cols, a->cols, sizeof(int) * nb, cudaMemcpyDeviceToDevice, st));
        if (d_values) CC(cudaMemcpyAsync(d_values, a->vals, sizeof(double) * 9 * nb, cudaMemcpyDeviceToDevice, st));
    }
    if (a->nact) {
        if (d_active) CC(cudaMemcpyAsync(d_active, a->act, sizeof(int) * a->nact, cudaMemcpyDeviceToDevice, st));
        if (d_E)
            CC(cudaMemcpyAsync(d_E, a->E, sizeof(double) * 12 * (size_t)a->nbody * a->nact, cudaMemcpyDeviceToDevice,
                               st));
    }
    return HSC_OK;
}

}  // extern "C"
