// Forward-mode derivatives (tangents) of the fused simulation step: the forward kernel
// instantiated with dual numbers, so that every quantity of the step carries its
// derivative along one input direction. The solve of the implicit system then gives
// the tangent of the voltage, A^{-1} (d rhs - dA v'), as the reference's forward-mode
// rule of the tree solve does (`_DHSSolveForwardAD`, solver_voltage.py:190-224), and
// the channels, stimulus, clamps and recordings carry theirs.
#include <cuda_runtime.h>
#include <stdio.h>

#include <mutex>

#include "jxb.h"
#include "jxb_sim_kernels.cuh"

namespace jxb {

namespace {

template <typename T>
SimKernel tangent_kernel(int threads, bool gm) {
  typedef Dual<T> D;
  if (threads <= 256) return gm ? sim_forward_kernel<D, 256, 1, true, false> : sim_forward_kernel<D, 256, 1, false, false>;
  return gm ? sim_forward_kernel<D, 512, 1, true, false> : sim_forward_kernel<D, 512, 1, false, false>;
}

std::mutex g_tangent_mu;
const void* g_tangent_granted[2][2][2];
size_t g_tangent_bytes[2][2][2];

}  // namespace

template <typename T>
static int launch_tangent(const JxbSimArgs& a, cudaStream_t stream) {
  typedef Dual<T> D;
  const size_t need = sim_smem_layout<D>(a, false, nullptr, nullptr);
  const bool gm = a.gscratch != nullptr;
  if (gm) {
    if (((uintptr_t)a.gscratch & 255) != 0 || a.gscratch_stride <= 0 || (a.gscratch_stride & 255) != 0 ||
        (size_t)a.gscratch_stride < need) {
      snprintf(g_err, sizeof(g_err),
               "gscratch must be 256-byte aligned with a stride (multiple of 256) of at least %zu bytes", need);
      return JXB_ERR_ARG;
    }
  } else if (need > 227 * 1024) {
    snprintf(g_err, sizeof(g_err), "work item needs %zu bytes of shared memory", need);
    return JXB_ERR_SMEM;
  }
  const int threads = a.threads > 0 ? a.threads : 256;
  if (threads % 32 != 0 || threads > 512) {
    snprintf(g_err, sizeof(g_err), "tangent launches take a multiple of 32 threads up to 512");
    return JXB_ERR_ARG;
  }
  SimKernel kern = tangent_kernel<T>(threads, gm);
  const size_t smem = gm ? 0 : need;
  {
    std::lock_guard<std::mutex> lock(g_tangent_mu);
    const int ti = sizeof(T) == 8, ni = threads > 256, gi = gm;
    if (g_tangent_granted[ti][ni][gi] != (const void*)kern || g_tangent_bytes[ti][ni][gi] < smem) {
      cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) {
        set_err("cudaFuncSetAttribute", e);
        return JXB_ERR_LAUNCH;
      }
      g_tangent_granted[ti][ni][gi] = (const void*)kern;
      g_tangent_bytes[ti][ni][gi] = smem;
    }
  }
  kern<<<a.n_items, threads, smem, stream>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("sim_forward_kernel (tangent)", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

int check_sim_args_public(const JxbSimArgs* a, bool backward);

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_sim_tangent(const JxbSimArgs* a, void* stream) {
  int rc = check_sim_args_public(a, false);
  if (rc != JXB_OK || a->n_items <= 0) return rc;
  if (a->multi || a->traj || a->traj_piv || a->syn_lin || a->syn_const) {
    snprintf(g_err, sizeof(g_err), "tangent launches run one problem without trajectory stores or synapses");
    return JXB_ERR_ARG;
  }
  // Every (value, tangent) array starts on a multiple of its pair size.
  const uintptr_t pair = a->dtype == JXB_F32 ? 8 : 16;
  const void* arrays[] = {a->a_low, a->a_up, a->gsum, a->cm, a->pbase, a->pscale, a->area,
                          a->stim, a->clamp, a->state, a->rec_out, a->ckpt};
  for (const void* p : arrays) {
    if (((uintptr_t)p) % pair != 0) {
      snprintf(g_err, sizeof(g_err), "tangent arrays must be aligned to %d bytes", (int)pair);
      return JXB_ERR_ARG;
    }
  }
  if (a->dtype == JXB_F32) return launch_tangent<float>(*a, (cudaStream_t)stream);
  return launch_tangent<double>(*a, (cudaStream_t)stream);
}

extern "C" int64_t jxb_sim_tangent_smem_bytes(const JxbSimArgs* a) {
  if (!a) return -1;
  if (a->dtype == JXB_F32) return (int64_t)sim_smem_layout<Dual<float>>(*a, false, nullptr, nullptr);
  return (int64_t)sim_smem_layout<Dual<double>>(*a, false, nullptr, nullptr);
}
