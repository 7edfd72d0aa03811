// Mixed-precision ray-patch intersection kernels of spheres and skin cells, compiled with fused
// multiply-adds (the build gives this file --fmad=true; every other device file, the mixed torus
// kernels of trace_mixed_torus.cu included, is compiled with --fmad=false).
#include "isect.cuh"

namespace nsg {

template <int PN>
void launch_isect_mixed_sphere(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                               cudaStream_t s) {
  k_isect_mixed<PN, false><<<sm_count() * tp.isect_bpsm, tp.isect_threads, 0, s>>>(C, co, hs);
}

template <int PN>
void launch_isect_quad_mixed(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                             cudaStream_t s) {
  k_isect_quad_mixed<PN><<<sm_count() * tp.isect_bpsm, tp.isect_threads, 0, s>>>(C, co, hs);
}

template void launch_isect_quad_mixed<0>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                         cudaStream_t);
template void launch_isect_quad_mixed<1>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                         cudaStream_t);
template void launch_isect_quad_mixed<2>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                         cudaStream_t);
template void launch_isect_mixed_sphere<0>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                           cudaStream_t);
template void launch_isect_mixed_sphere<1>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                           cudaStream_t);
template void launch_isect_mixed_sphere<2>(const TraceCtx&, const CandOut&, const HitStore&, const TuneParams&,
                                           cudaStream_t);

}  // namespace nsg
