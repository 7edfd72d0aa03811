// Mixed-precision torus intersection kernels, compiled without fused multiply-adds like the
// double-precision path: their clipping-sphere entry and quartic solve repeat the FP64 path's
// operations (only the feasibility tests run in FP32), so that the reference's solver, which is
// ill-conditioned for some rays, returns the same roots in both precisions.
#include "isect.cuh"

namespace nsg {

template <int PN>
void launch_isect_mixed_torus(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                              cudaStream_t s) {
  k_isect_mixed<PN, true><<<sm_count() * tp.isect_bpsm, tp.isect_threads, 0, s>>>(C, co, hs);
}

template void launch_isect_mixed_torus<0>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                          cudaStream_t);
template void launch_isect_mixed_torus<1>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                          cudaStream_t);
template void launch_isect_mixed_torus<2>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                          cudaStream_t);

}  // namespace nsg
