// Numeric status of a factorization: kernels OR these bits into the handle's
// device status word (the task descriptors carry its address); the host reads
// it once the factorization is done and reports SPQ_ERR_NUMERIC.
#pragma once
#include "kernels.hpp"

namespace spq {

// A Householder pivot of an elimination or scaling QR: R_kk non-finite (NaN or
// Inf reached the factor) or exactly zero (the stacked column, or the
// interface's diagonal block, is singular).
template <class T>
__device__ __forceinline__ void note_qr_pivot(int* status, T beta) {
    if (!status) return;
    if (!isfinite(beta))
        atomicOr(status, kStatNonFinite);
    else if (beta == T(0))
        atomicOr(status, kStatZeroPivot);
}

// A pivot step of the truncated RRQR of a sparsification: a non-finite R_kk,
// or no column left with a finite norm before the rank rule stopped the
// factorization (NaN in the interface's blocks).
template <class T>
__device__ __forceinline__ void note_rrqr_pivot(int* status, T beta) {
    if (status && !isfinite(beta)) atomicOr(status, kStatNonFinite);
}
__device__ __forceinline__ void note_rrqr_nan(int* status) {
    if (status) atomicOr(status, kStatNonFinite | kStatRRQRNaN);
}

}  // namespace spq
