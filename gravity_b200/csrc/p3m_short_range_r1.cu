// p3m_short_range_r1.cu — short-range kernels with a stencil half-width of
// 1 cell(s) in x (see p3m_short_range.cuh).
#include "p3m_short_range.cuh"

namespace p3m {
P3M_DEFINE_SHORT_RANGE_RX(1)
}  // namespace p3m
