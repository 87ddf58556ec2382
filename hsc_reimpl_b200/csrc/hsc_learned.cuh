// Learned polynomial preconditioner (hsc_learned.cu): per-system spectral
// features computed on the device and the 16-64-64-8 MLP that maps them to
// the Schur-basis polynomial weights, evaluated inside a solve.
#pragma once
#include <cstdint>

#include "hsc_internal.cuh"

namespace hsc {

constexpr int kFeat = 16;      // MLP inputs
constexpr int kHidden = 64;    // two hidden layers
constexpr int kPolyOut = 8;    // positive polynomial weights
// flat parameter layout, row-major (out x in): W1, b1, W2, b2, W3, b3
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kFeat;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kPolyOut * kHidden;
constexpr int kParams = kOffB3 + kPolyOut;  // 5768

// previous-solve record of one system, kept on the device next to its scalars
//   [0] 1 if a previous solve exists, [1] lambda_min, [2] lambda_max of its
//   preconditioned Schur operator (Lanczos), [3] its PCG iterations,
//   [4] q(0) = sum of its polynomial weights (so lambda_min / q(0) estimates
//   the smallest eigenvalue of w Dd^-1 S), [5] unused
constexpr int kPrev = 6;
constexpr int kFeatParts = 16;  // doubles per block partial of the row statistics

struct FeatArgs {
    int n, nnz, a, kmax;
    const int* rowptr;
    const int* colidx;
    const int* diag_pos;
    const int* rowflag;
    const double* v64;         // FP64 BSR planes of D, element e of block k at v64[e * nnz + k]
    const int* rank;           // device scalar
    const double* vt64;        // Vt (a x kmax, column-major)
    const double* dpiv;        // LDL^T pivots
    const double* prev;        // kPrev doubles
    const uint16_t* mlp;       // BF16 parameters, or null: features only
    float* feat;               // out: kFeat
    double* w;                 // out: kPolyOut weights (when mlp)
    double* part;              // scratch: nparts x kFeatParts
    int nparts;
};

cudaError_t launch_features(const FeatArgs& f, cudaStream_t st);

}  // namespace hsc
