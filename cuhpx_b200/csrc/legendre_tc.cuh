// Tensor-core (tcgen05) Legendre contraction for mixed-precision plans.
// Placeholder: mixed-precision plans are rejected until the kernels land.
#pragma once

#include "legendre.cuh"

namespace hpx {

struct TcPlan {
    int active = 0;
};

inline const char* tc_last_error() { return "tensor-core contraction not built"; }
inline int tc_create(TcPlan&, int, int, int, int, int, int) { return 5; }
inline void tc_release(TcPlan&) {}
inline size_t tc_workspace_bytes(const TcPlan&) { return 0; }
inline void tc_forward(const TcPlan&, const float*, int, int, float*, int, int, int, const RingPair*, const int*,
                       const double2*, int, cudaStream_t) {}
inline void tc_inverse(const TcPlan&, const float*, int, float*, int, int, int, const RingPair*, const int*,
                       const double2*, const int2*, int, cudaStream_t) {}

}  // namespace hpx
