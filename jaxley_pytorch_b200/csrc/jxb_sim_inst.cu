// Instantiations of the fused simulation kernels for one element type, kind and CTA
// size class. The build compiles this unit once per combination, defining
//   JXB_INST_T    float or double
//   JXB_INST_BWD  0 forward, 1 adjoint
//   JXB_INST_NT   256, 384, 512 or 1024 (threads per CTA the kernels are bounded for)
//   JXB_INST_FN   the name of the selector it defines (declared in jxb_sim_kernels.cuh)
// so that the instantiations compile in parallel.
#include "jxb_sim_kernels.cuh"

#if !defined(JXB_INST_T) || !defined(JXB_INST_BWD) || !defined(JXB_INST_NT) || !defined(JXB_INST_FN)
#error "jxb_sim_inst.cu is compiled with JXB_INST_T, JXB_INST_BWD, JXB_INST_NT and JXB_INST_FN"
#endif

namespace jxb {
namespace {

using T = JXB_INST_T;
constexpr bool kBwd = JXB_INST_BWD != 0;
constexpr int kNT = JXB_INST_NT;

template <int MINB, bool GM, bool MULTI>
SimKernel one() {
  if constexpr (kBwd)
    return sim_backward_kernel<T, kNT, MINB, GM, MULTI>;
  else
    return sim_forward_kernel<T, kNT, MINB, GM, MULTI>;
}

}  // namespace

SimKernel JXB_INST_FN(bool gm, bool multi, bool wide) {
  if (wide) {
    // float, up to 256 threads: two CTAs per SM with up to 128 registers a thread
    if constexpr (sizeof(T) == 4 && kNT == 256) {
      if (multi) return nullptr;
      return gm ? one<2, true, false>() : one<2, false, false>();
    }
    return nullptr;
  }
  constexpr int B = kMinBlocks<T, kNT>;
  if (multi) return gm ? one<B, true, true>() : one<B, false, true>();
  return gm ? one<B, true, false>() : one<B, false, false>();
}

}  // namespace jxb
