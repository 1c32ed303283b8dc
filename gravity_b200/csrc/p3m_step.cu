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
