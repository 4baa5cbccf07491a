// dispatch.cuh — map the runtime (precision, reals-per-link) pair of a lattice onto the
// four compiled storage variants.
#pragma once
#include "kernels.h"

#define QCB_PREC_FP64 0
#define QCB_PREC_FP32 1

// Evaluates to the return of FN<S, NR>(args...) for the lattice's storage variant.
#define QCB_DISPATCH_STORE(L, FN, ...)                                             \
  do {                                                                           \
    switch ((L).prec * 100 + (L).nr) {                                           \
      case QCB_PREC_FP64 * 100 + 18:                                             \
        return FN<double, 18>(__VA_ARGS__);                                      \
      case QCB_PREC_FP64 * 100 + 12:                                             \
        return FN<double, 12>(__VA_ARGS__);                                      \
      case QCB_PREC_FP32 * 100 + 18:                                             \
        return FN<float, 18>(__VA_ARGS__);                                       \
      case QCB_PREC_FP32 * 100 + 12:                                             \
        return FN<float, 12>(__VA_ARGS__);                                       \
      default:                                                                   \
        return cudaErrorInvalidValue;                                            \
    }                                                                            \
  } while (0)

namespace qcb {
inline unsigned grid_for(uint64_t n, int block) { return (unsigned)((n + (uint64_t)block - 1) / (uint64_t)block); }
}  // namespace qcb
