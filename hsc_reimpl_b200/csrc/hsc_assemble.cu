// GPU assembly of the log-Neo-Hookean Tet4 Hessian into the solver's input
// form (one-triangle BCOO of 3x3 blocks, sorted and unique, column-major
// values) -- the producer of the FEM block of each Newton system, so a
// simulation can hand the solver its matrix without a host round trip.
//
// Per tet (reference: log_neo_hookean_3d.cu:62-135 and
// log_neo_hookean_function.h:77-150):
//   F = Ds Dm^-1,  H9 = mu I + lambda vec(G) vec(G)^T - q T(G),  G = cof(F)/J,
//   q = lambda ln J - mu  (column-major vec(F), element F[i][a] at 3a + i);
//   H9 projected to SPD by a cyclic Jacobi eigen-decomposition with negative
//   eigenvalues clamped to 0;  scaled by V dt^2;  pulled back to the ten node
//   blocks (a, b) = sum_ij Gs[a][i] Gs[b][j] H9[i-th 3x3 column block ...] of
//   the upper triangle (node(a) <= node(b)), as the reference writes them.
// The lumped mass rho V / 4 per incident tet is added to the diagonal blocks.
//
// Determinism: the per-tet blocks go to a staging array; each BCOO block sums
// its contributions in a fixed (tet, slot) order from a CSR list built once
// per mesh -- no floating-point atomics (the reference's triplet assembly sums
// duplicates in sort order).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/hsc_c_api.h"
#include "hsc_internal.cuh"

namespace hsc {
namespace {

constexpr int kSlots = 10;  // upper node-pair blocks of a Tet4

__device__ __forceinline__ double det3(const double* m) {  // row-major 3x3
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// cofactor matrix (row-major): C[i][j] = (-1)^(i+j) minor(i, j)
__device__ __forceinline__ void cof3(const double* F, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            C[3 * i + j] = F[3 * i1 + j1] * F[3 * i2 + j2] - F[3 * i1 + j2] * F[3 * i2 + j1];
        }
}

// symmetric 9x9 (row-major) -> its projection onto the PSD cone: cyclic Jacobi
// rotations until every off-diagonal entry is below 1e-13 |H|_F (at most 32
// sweeps), eigenvalues clamped at 0, H = Q diag(max(l, 0)) Q^T
__device__ void project_psd9(double* H) {
    double Q[81];
    for (int i = 0; i < 81; ++i) Q[i] = (i % 10 == 0) ? 1.0 : 0.0;
    double nrm = 0.0;
    for (int i = 0; i < 81; ++i) nrm += H[i] * H[i];
    const double thr = 1e-13 * sqrt(nrm);
    for (int sweep = 0; sweep < 32; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 8; ++p)
            for (int q = p + 1; q < 9; ++q) {
                const double apq = H[9 * p + q];
                off = fmax(off, fabs(apq));
                if (fabs(apq) <= thr) continue;
                const double theta = (H[9 * q + q] - H[9 * p + p]) / (2.0 * apq);
                const double t = copysign(1.0 / (fabs(theta) + sqrt(1.0 + theta * theta)), theta);
                const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                H[9 * p + p] -= t * apq;
                H[9 * q + q] += t * apq;
                H[9 * p + q] = H[9 * q + p] = 0.0;
                for (int k = 0; k < 9; ++k) {
                    if (k != p && k != q) {
                        const double kp = H[9 * k + p], kq = H[9 * k + q];
                        H[9 * k + p] = H[9 * p + k] = c * kp - s * kq;
                        H[9 * k + q] = H[9 * q + k] = s * kp + c * kq;
                    }
                    const double qp = Q[9 * k + p], qq = Q[9 * k + q];
                    Q[9 * k + p] = c * qp - s * qq;
                    Q[9 * k + q] = s * qp + c * qq;
                }
            }
        if (off <= thr) break;
    }
    double lam[9];
    for (int i = 0; i < 9; ++i) lam[i] = fmax(H[10 * i], 0.0);
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) {
            double v = 0.0;
            for (int k = 0; k < 9; ++k) v += Q[9 * i + k] * lam[k] * Q[9 * j + k];
            H[9 * i + j] = v;
        }
}

// one thread per tet: the ten upper blocks, column-major, into stage[tet][slot][9]
__global__ void tet_hessian_kernel(const int* __restrict__ tets, int ntet, const double* __restrict__ x,
                                   const double* __restrict__ dminv, const double* __restrict__ vol,
                                   const double* __restrict__ E, double nu, double dt, int project,
                                   double* __restrict__ stage, int* bad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntet) return;
    const int nd[4] = {tets[4 * t], tets[4 * t + 1], tets[4 * t + 2], tets[4 * t + 3]};
    const double* Dm = dminv + 9 * (size_t)t;  // Dm^-1, row-major
    double Ds[9];                              // columns: x1 - x0, x2 - x0, x3 - x0
    for (int i = 0; i < 3; ++i)
        for (int c = 0; c < 3; ++c) Ds[3 * i + c] = x[3 * (size_t)nd[c + 1] + i] - x[3 * (size_t)nd[0] + i];
    double F[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            F[3 * i + j] = Ds[3 * i] * Dm[j] + Ds[3 * i + 1] * Dm[3 + j] + Ds[3 * i + 2] * Dm[6 + j];
    const double J = det3(F);
    double* out = stage + (size_t)t * kSlots * 9;
    if (!(J > 0.0) || !isfinite(J)) {
        atomicAdd(bad, 1);
        for (int e = 0; e < kSlots * 9; ++e) out[e] = 0.0;
        return;
    }
    const double Et = E[t];
    const double mu = Et / (2.0 * (1.0 + nu)), lam = Et * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double C[9], G[9];
    cof3(F, C);
    for (int e = 0; e < 9; ++e) G[e] = C[e] / J;
    const double q = lam * log(J) - mu;
    double H[81];
    // H[i + 3a][j + 3b] = mu d_ij d_ab + lam G[i][a] G[j][b] - q G[i][b] G[j][a]
    for (int a = 0; a < 3; ++a)
        for (int i = 0; i < 3; ++i)
            for (int b = 0; b < 3; ++b)
                for (int j = 0; j < 3; ++j)
                    H[9 * (i + 3 * a) + (j + 3 * b)] = ((i == j && a == b) ? mu : 0.0) +
                                                       lam * G[3 * i + a] * G[3 * j + b] -
                                                       q * G[3 * i + b] * G[3 * j + a];
    if (project) project_psd9(H);
    const double s = vol[t] * dt * dt;
    // shape gradients: Gs[k][a], k = 0..3 nodes; F[i][a] = sum_k x_k[i] Gs[k][a]
    double Gs[12];
    for (int a = 0; a < 3; ++a) {
        Gs[a] = -(Dm[a] + Dm[3 + a] + Dm[6 + a]);
        for (int k = 1; k < 4; ++k) Gs[3 * k + a] = Dm[3 * (k - 1) + a];
    }
    int slot = 0;
    for (int u = 0; u < 4; ++u)
        for (int v = u; v < 4; ++v, ++slot) {
            // upper block (node order): rows of the smaller node id
            const int L = nd[u] <= nd[v] ? u : v, R = nd[u] <= nd[v] ? v : u;
            double* blk = out + 9 * slot;
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    double acc = 0.0;
                    for (int a = 0; a < 3; ++a)
                        for (int b = 0; b < 3; ++b) acc += Gs[3 * L + a] * Gs[3 * R + b] * H[9 * (i + 3 * a) + (j + 3 * b)];
                    blk[i + 3 * j] = s * acc;  // column-major: (i, j) at i + 3 j
                }
        }
}

// one thread per BCOO block: the staged contributions in (tet, slot) order, plus the lumped mass
__global__ void gather_blocks_kernel(const int* __restrict__ ptr, const int* __restrict__ src, int nblk,
                                     const double* __restrict__ stage, const double* __restrict__ mass,
                                     const int* __restrict__ rows, const int* __restrict__ cols,
                                     double* __restrict__ values) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nblk) return;
    double acc[9];
    for (int e = 0; e < 9; ++e) acc[e] = 0.0;
    for (int p = ptr[k]; p < ptr[k + 1]; ++p) {
        const double* b = stage + 9 * (size_t)src[p];
        for (int e = 0; e < 9; ++e) acc[e] += b[e];
    }
    if (rows[k] == cols[k]) {
        const double m = mass[rows[k]];
        acc[0] += m; acc[4] += m; acc[8] += m;
    }
    double* o = values + 9 * (size_t)k;
    for (int e = 0; e < 9; ++e) o[e] = acc[e];
}

// ---------------------------------------------------------------------------
// line-search feasibility (reference: feasible_segment, log_neo_hookean_function.h:37-75,
// applied per tet in the energy kernel, log_neo_hookean_3d.cu:45-52, so a trial
// step whose segment inverts a tet has infinite energy and the search halves it)
// ---------------------------------------------------------------------------
constexpr double kMinJacobian = 1e-8;

__device__ __forceinline__ double triple3(const double* A, int c0, const double* B, int c1, const double* C, int c2) {
    // a . (b x c) for column c0 of A, c1 of B, c2 of C (row-major 3x3)
    const double a0 = A[c0], a1 = A[3 + c0], a2 = A[6 + c0];
    const double b0 = B[c1], b1 = B[3 + c1], b2 = B[6 + c1];
    const double d0 = C[c2], d1 = C[3 + c2], d2 = C[6 + c2];
    return a0 * (b1 * d2 - b2 * d1) + a1 * (b2 * d0 - b0 * d2) + a2 * (b0 * d1 - b1 * d0);
}

// det(A + s (E - A)) > min_jacobian for every s in [0, 1]: the endpoints and the
// roots of the derivative of the cubic, which hold its interior minima
__device__ bool segment_feasible(const double* A, const double* E) {
    double B[9];
    for (int e = 0; e < 9; ++e) B[e] = E[e] - A[e];
    const double c0 = det3(A);
    const double c1 = triple3(B, 0, A, 1, A, 2) + triple3(A, 0, B, 1, A, 2) + triple3(A, 0, A, 1, B, 2);
    const double c2 = triple3(A, 0, B, 1, B, 2) + triple3(B, 0, A, 1, B, 2) + triple3(B, 0, B, 1, A, 2);
    const double c3 = det3(B);
    if (!(c0 > kMinJacobian && det3(E) > kMinJacobian)) return false;
    const double a = 3.0 * c3, b = 2.0 * c2, c = c1;
    double roots[2] = {-1.0, -1.0};
    const double scale = fabs(a) + fabs(b) + fabs(c);
    const double eps = 32.0 * 2.220446049250313e-16 * scale;
    if (fabs(a) <= eps) {
        if (fabs(b) > eps) roots[0] = -c / b;
    } else {
        const double disc = b * b - 4.0 * a * c;
        if (disc >= 0.0) {
            const double q = -0.5 * (b + copysign(sqrt(disc), b));
            if (q == 0.0) roots[0] = -b / (2.0 * a);
            else { roots[0] = q / a; roots[1] = c / q; }
        }
    }
    for (int i = 0; i < 2; ++i) {
        const double s = roots[i];
        if (s > 0.0 && s < 1.0 && !(((c3 * s + c2) * s + c1) * s + c0 > kMinJacobian)) return false;
    }
    return true;
}

// per tet: the fewest halvings m of alpha0 whose trial segment is feasible
// (max_halvings + 1 when none is); the step is set by the worst tet
__global__ void feasible_step_kernel(const int* __restrict__ tets, int ntet, const double* __restrict__ x0,
                                     const double* __restrict__ dx, const double* __restrict__ dminv, double alpha0,
                                     int max_halvings, int* worst, int* count) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntet) return;
    const int nd[4] = {tets[4 * t], tets[4 * t + 1], tets[4 * t + 2], tets[4 * t + 3]};
    const double* Dm = dminv + 9 * (size_t)t;
    auto defgrad = [&](double s, double* F) {  // F at x0 + s dx
        double Ds[9];
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 3; ++c) {
                const size_t a = 3 * (size_t)nd[c + 1] + i, o = 3 * (size_t)nd[0] + i;
                Ds[3 * i + c] = (x0[a] + s * dx[a]) - (x0[o] + s * dx[o]);
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                F[3 * i + j] = Ds[3 * i] * Dm[j] + Ds[3 * i + 1] * Dm[3 + j] + Ds[3 * i + 2] * Dm[6 + j];
    };
    double F0[9], F1[9];
    defgrad(0.0, F0);
    int m = 0;
    double s = alpha0;
    for (; m <= max_halvings; ++m, s *= 0.5) {
        defgrad(s, F1);
        if (segment_feasible(F0, F1)) break;
    }
    if (m > 0) {
        atomicMax(worst, m);
        atomicAdd(count, 1);
    }
}

}  // namespace
}  // namespace hsc

struct hsc_fem_assembler {
    int ntet = 0, nnode = 0, nblk = 0;
    double nu = 0.3, dt = 1.0 / 30.0;
    int project = 1;
    int* tets = nullptr;       // device ntet x 4
    double* dminv = nullptr;   // device ntet x 9
    double* vol = nullptr;     // device ntet
    double* mass = nullptr;    // device nnode
    int* rows = nullptr;       // device nblk
    int* cols = nullptr;
    int* ptr = nullptr;        // device nblk + 1
    int* src = nullptr;        // device ntet x 10
    double* stage = nullptr;   // device ntet x 10 x 9
    int* bad = nullptr;        // device counter of inverted tets / worst halving count
    int* aux = nullptr;        // device counter of tets that limit the step
};

namespace {
void free_assembler(hsc_fem_assembler* a) {
    if (!a) return;
    cudaFree(a->tets); cudaFree(a->dminv); cudaFree(a->vol); cudaFree(a->mass); cudaFree(a->rows);
    cudaFree(a->cols); cudaFree(a->ptr); cudaFree(a->src); cudaFree(a->stage); cudaFree(a->bad); cudaFree(a->aux);
    delete a;
}
template <class T> cudaError_t upload(T** d, const std::vector<T>& h) {
    cudaError_t e = cudaMalloc((void**)d, sizeof(T) * std::max<size_t>(1, h.size()));
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return e;
}
}  // namespace

extern "C" {

int hsc_fem_assembler_create(const int32_t* tets, int32_t ntet, int32_t nnode, const double* rest_x, double rho,
                             double nu, double dt, int32_t project, hsc_fem_assembler** out) {
    if (!tets || !rest_x || !out || ntet < 1 || nnode < 1 || !(rho > 0) || !(nu > -1 && nu < 0.5) || !(dt > 0))
        return HSC_ERR_INVALID;
    *out = nullptr;
    std::vector<double> dminv(9 * (size_t)ntet), vol(ntet), mass(nnode, 0.0);
    for (int t = 0; t < ntet; ++t) {
        int nd[4];
        for (int k = 0; k < 4; ++k) {
            nd[k] = tets[4 * t + k];
            if (nd[k] < 0 || nd[k] >= nnode) return HSC_ERR_INVALID;
        }
        double Dm[9];  // row-major, columns = edges x_k - x_0
        for (int i = 0; i < 3; ++i)
            for (int c = 0; c < 3; ++c) Dm[3 * i + c] = rest_x[3 * (size_t)nd[c + 1] + i] - rest_x[3 * (size_t)nd[0] + i];
        const double det = Dm[0] * (Dm[4] * Dm[8] - Dm[5] * Dm[7]) - Dm[1] * (Dm[3] * Dm[8] - Dm[5] * Dm[6]) +
                           Dm[2] * (Dm[3] * Dm[7] - Dm[4] * Dm[6]);
        if (!(std::fabs(det) > 0)) return HSC_ERR_INVALID;
        double inv[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
                inv[3 * i + j] = (Dm[3 * i1 + j1] * Dm[3 * i2 + j2] - Dm[3 * i1 + j2] * Dm[3 * i2 + j1]) / det;
            }
        std::memcpy(&dminv[9 * (size_t)t], inv, sizeof inv);
        vol[t] = std::fabs(det) / 6.0;
        for (int k = 0; k < 4; ++k) mass[nd[k]] += rho * vol[t] / 4.0;
    }
    // the upper-triangle block pattern and, per block, its (tet, slot) contributions in order
    std::vector<long long> key((size_t)ntet * hsc::kSlots);
    for (int t = 0; t < ntet; ++t) {
        int slot = 0;
        for (int u = 0; u < 4; ++u)
            for (int v = u; v < 4; ++v, ++slot) {
                const long long a = tets[4 * t + u], b = tets[4 * t + v];
                key[(size_t)t * hsc::kSlots + slot] = std::min(a, b) * nnode + std::max(a, b);
            }
    }
    std::vector<long long> uk(key);
    for (int i = 0; i < nnode; ++i) uk.push_back((long long)i * nnode + i);  // every node's diagonal block
    std::sort(uk.begin(), uk.end());
    uk.erase(std::unique(uk.begin(), uk.end()), uk.end());
    const int nblk = (int)uk.size();
    std::vector<int> rows(nblk), cols(nblk), ptr(nblk + 1, 0), src((size_t)ntet * hsc::kSlots);
    for (int k = 0; k < nblk; ++k) { rows[k] = (int)(uk[k] / nnode); cols[k] = (int)(uk[k] % nnode); }
    std::vector<int> bidx(key.size());
    for (size_t e = 0; e < key.size(); ++e) {
        bidx[e] = (int)(std::lower_bound(uk.begin(), uk.end(), key[e]) - uk.begin());
        ++ptr[bidx[e] + 1];
    }
    for (int k = 0; k < nblk; ++k) ptr[k + 1] += ptr[k];
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (size_t e = 0; e < key.size(); ++e) src[fill[bidx[e]]++] = (int)e;  // e ascending: (tet, slot) order
    hsc_fem_assembler* a = new hsc_fem_assembler();
    a->ntet = ntet; a->nnode = nnode; a->nblk = nblk; a->nu = nu; a->dt = dt; a->project = project ? 1 : 0;
    std::vector<int> tv(tets, tets + 4 * (size_t)ntet);
    cudaError_t e = upload(&a->tets, tv);
    if (e == cudaSuccess) e = upload(&a->dminv, dminv);
    if (e == cudaSuccess) e = upload(&a->vol, vol);
    if (e == cudaSuccess) e = upload(&a->mass, mass);
    if (e == cudaSuccess) e = upload(&a->rows, rows);
    if (e == cudaSuccess) e = upload(&a->cols, cols);
    if (e == cudaSuccess) e = upload(&a->ptr, ptr);
    if (e == cudaSuccess) e = upload(&a->src, src);
    if (e == cudaSuccess) e = cudaMalloc((void**)&a->stage, sizeof(double) * 9 * hsc::kSlots * (size_t)ntet);
    if (e == cudaSuccess) e = cudaMalloc((void**)&a->bad, sizeof(int));
    if (e != cudaSuccess) { free_assembler(a); return e == cudaErrorMemoryAllocation ? HSC_ERR_ALLOC : HSC_ERR_CUDA; }
    *out = a;
    return HSC_OK;
}

void hsc_fem_assembler_destroy(hsc_fem_assembler* a) { free_assembler(a); }

int hsc_fem_pattern(const hsc_fem_assembler* a, int32_t* d_rows, int32_t* d_cols, int64_t* nnzb) {
    if (!a) return HSC_ERR_INVALID;
    if (nnzb) *nnzb = a->nblk;
    if (d_rows && cudaMemcpy(d_rows, a->rows, sizeof(int) * a->nblk, cudaMemcpyDeviceToDevice) != cudaSuccess)
        return HSC_ERR_CUDA;
    if (d_cols && cudaMemcpy(d_cols, a->cols, sizeof(int) * a->nblk, cudaMemcpyDeviceToDevice) != cudaSuccess)
        return HSC_ERR_CUDA;
    return HSC_OK;
}

int hsc_fem_assemble(hsc_fem_assembler* a, const double* d_x, const double* d_E, double* d_values,
                     int32_t* inverted, void* stream) {
    if (!a || !d_x || !d_E || !d_values) return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(a->bad, 0, sizeof(int), st) != cudaSuccess) return HSC_ERR_CUDA;
    hsc::count_launch();
    hsc::tet_hessian_kernel<<<(a->ntet + 127) / 128, 128, 0, st>>>(a->tets, a->ntet, d_x, a->dminv, a->vol, d_E, a->nu,
                                                                  a->dt, a->project, a->stage, a->bad);
    hsc::count_launch();
    hsc::gather_blocks_kernel<<<(a->nblk + 255) / 256, 256, 0, st>>>(a->ptr, a->src, a->nblk, a->stage, a->mass, a->rows,
                                                                    a->cols, d_values);
    if (cudaGetLastError() != cudaSuccess) return HSC_ERR_CUDA;
    if (inverted) {
        if (cudaMemcpyAsync(inverted, a->bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HSC_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return HSC_ERR_CUDA;
        if (*inverted) return HSC_ERR_NONSPD;
    }
    return HSC_OK;
}

int hsc_fem_feasible_step(hsc_fem_assembler* a, const double* d_x0, const double* d_dx, double alpha0,
                          int32_t max_halvings, double* alpha, int32_t* halvings, int32_t* limited, void* stream) {
    if (!a || !d_x0 || !d_dx || !alpha || !(alpha0 > 0) || max_halvings < 0 || max_halvings > 1000)
        return HSC_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(a->bad, 0, sizeof(int), st) != cudaSuccess) return HSC_ERR_CUDA;
    if (!a->aux && cudaMalloc((void**)&a->aux, sizeof(int)) != cudaSuccess) return HSC_ERR_ALLOC;
    if (cudaMemsetAsync(a->aux, 0, sizeof(int), st) != cudaSuccess) return HSC_ERR_CUDA;
    hsc::count_launch();
    hsc::feasible_step_kernel<<<(a->ntet + 127) / 128, 128, 0, st>>>(a->tets, a->ntet, d_x0, d_dx, a->dminv, alpha0,
                                                                    max_halvings, a->bad, a->aux);
    if (cudaGetLastError() != cudaSuccess) return HSC_ERR_CUDA;
    int h[2] = {0, 0};
    if (cudaMemcpyAsync(&h[0], a->bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HSC_ERR_CUDA;
    if (cudaMemcpyAsync(&h[1], a->aux, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HSC_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HSC_ERR_CUDA;
    if (halvings) *halvings = h[0];
    if (limited) *limited = h[1];
    if (h[0] > max_halvings) { *alpha = 0.0; return HSC_ERR_NONSPD; }
    *alpha = std::ldexp(alpha0, -h[0]);
    return HSC_OK;
}

}  // extern "C"
