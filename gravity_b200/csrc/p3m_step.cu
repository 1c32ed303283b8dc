// p3m_step.cu — the stages of the P3M step as one translation unit: the cell
// and Morton sorts, the drift, the deposit, the real FFT with the Green's
// multiply, interpolation + kick and the short range's dispatch (step/), and
// the persistent kernel of the batched form, which runs the batched bodies of
// all of them in a single launch (step/p3m_batch_persistent.cu).
#include "step/p3m_sort.cu"
#include "step/p3m_drift.cu"
#include "step/p3m_deposit.cu"
#include "step/p3m_fft.cu"
#include "step/p3m_kick.cu"

// The coherent copy of the stage bodies for the persistent kernel: the same
// sources inside namespace p3m::coherent, with every load through the
// ordinary (coherent) path -- no __ldg, no __restrict__ that would let the
// compiler use the read-only non-coherent one -- and without their host-side
// launchers. Within one persistent launch a stage reads what other SMs wrote
// in an earlier phase, which the non-coherent path may serve stale.
#define P3M_COHERENT_BODIES 1
#define __ldg(p) (*(p))
#define __restrict__
namespace p3m {
namespace coherent {
#include "p3m_short_range.cuh"
#include "step/p3m_sort.cu"
#include "step/p3m_drift.cu"
#include "step/p3m_deposit.cu"
#include "step/p3m_fft.cu"
#include "step/p3m_kick.cu"
}  // namespace coherent
}  // namespace p3m
#undef __restrict__
#undef __ldg
#undef P3M_COHERENT_BODIES

#include "step/p3m_batch_persistent.cu"
