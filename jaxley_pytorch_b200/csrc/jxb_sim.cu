// Fused bwd_euler + DHS simulation kernels (forward and adjoint).
//
// One CTA owns one work item: a block of whole trees (cells) and a few batch rows.
// Everything the step reads repeatedly is staged in shared memory when the launch
// starts: the block's node metadata, its chain schedule, the off-diagonal entries of
// the tree system, the channel programs, the rows' parameter values and the rows'
// state vectors, which stay resident for the whole segment of steps. Per step:
//   1. channels, node-parallel: gate updates in insertion order, linearised currents
//      (modules/base.py:3402-3542), stimulus (:3234-3242), assembly of the diagonal
//      and right-hand side of the implicit system (solver_voltage.py:250-291);
//   2. the Hines solve of every tree (solver_voltage.py:78-108), organised by chains
//      (a node and its only child share a chain): one thread eliminates a whole
//      chain bottom-up in registers, the chains of one level run in parallel and
//      levels are separated by a barrier; back-substitution runs the levels top-down.
// The adjoint kernel recomputes a segment from its checkpoint (storing the state
// before every step), then runs the steps in reverse: the transposed tree solve
// (the same chain schedule with the off-diagonals swapped, solver_voltage.py:143-187)
// and the vector-Jacobian products of the channel step, node by node.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "jxb.h"
#include "jxb_sim_kernels.cuh"

namespace jxb {

thread_local char g_err[512] = "";

void set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, e == cudaSuccess ? "ok" : cudaGetErrorString(e));
}


// The kernel instantiation of a launch (jxb_sim_inst.cu units).
template <typename T>
SimKernel pick_kernel(bool backward, int threads, bool gm, bool multi, bool wide) {
  const bool f = sizeof(T) == 4;
  if (threads <= 256) {
    if (f) return backward ? sim_kernel_f32_bwd_256(gm, multi, wide) : sim_kernel_f32_fwd_256(gm, multi, wide);
    return backward ? sim_kernel_f64_bwd_256(gm, multi, wide) : sim_kernel_f64_fwd_256(gm, multi, wide);
  }
  if (threads <= 384 && f && backward) return sim_kernel_f32_bwd_384(gm, multi, false);
  if (threads <= 512) {
    if (f) return backward ? sim_kernel_f32_bwd_512(gm, multi, false) : sim_kernel_f32_fwd_512(gm, multi, false);
    return backward ? sim_kernel_f64_bwd_512(gm, multi, false) : sim_kernel_f64_fwd_512(gm, multi, false);
  }
  if (f) return backward ? sim_kernel_f32_bwd_1024(gm, multi, false) : sim_kernel_f32_fwd_1024(gm, multi, false);
  return backward ? sim_kernel_f64_bwd_1024(gm, multi, false) : sim_kernel_f64_fwd_1024(gm, multi, false);
}

// Largest dynamic shared memory already granted to a kernel on a device:
// cudaFuncSetAttribute is called only when a launch needs more, so steady-state
// launches make no extra runtime call.
struct SmemGrant {
  const void* fn;
  int device;
  size_t bytes;
};
static SmemGrant g_grants[256];
static int g_n_grants = 0;
static std::mutex g_grants_mu;

static cudaError_t grant_smem(const void* fn, size_t smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_grants_mu);
  for (int i = 0; i < g_n_grants; ++i)
    if (g_grants[i].fn == fn && g_grants[i].device == dev) {
      if (g_grants[i].bytes >= smem) return cudaSuccess;
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e == cudaSuccess) g_grants[i].bytes = smem;
      return e;
    }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && g_n_grants < 256) g_grants[g_n_grants++] = {fn, dev, smem};
  return e;
}

template <typename T>
int launch_sim(const JxbSimArgs& a, bool backward, cudaStream_t stream) {
  const size_t need = sim_smem_layout<T>(a, backward, nullptr, nullptr);
  const bool gm = a.gscratch != nullptr;
  if (gm) {
    if (((uintptr_t)a.gscratch & 255) != 0 || a.gscratch_stride <= 0 || (a.gscratch_stride & 255) != 0 ||
        (size_t)a.gscratch_stride < need) {
      snprintf(g_err, sizeof(g_err),
               "gscratch must be 256-byte aligned with a stride (multiple of 256) of at least %zu bytes",
               need);
      return JXB_ERR_ARG;
    }
  } else if (need > 227 * 1024) {
    snprintf(g_err, sizeof(g_err), "work item needs %zu bytes of shared memory", need);
    return JXB_ERR_SMEM;
  }
  if (backward && a.gacc) {
    const size_t gneed = sizeof(T) * (size_t)a.max_rows * (size_t)a.max_gslots;
    if (((uintptr_t)a.gacc & 255) != 0 || a.gacc_stride <= 0 || (a.gacc_stride & 255) != 0 ||
        (size_t)a.gacc_stride < gneed) {
      snprintf(g_err, sizeof(g_err),
               "gacc must be 256-byte aligned with a stride (multiple of 256) of at least %zu bytes", gneed);
      return JXB_ERR_ARG;
    }
  }
  const size_t smem = gm ? 0 : need;
  const int threads = a.threads > 0 ? a.threads : 256;
  if (threads % 32 != 0 || threads > 1024) {
    snprintf(g_err, sizeof(g_err), "threads must be a multiple of 32 up to 1024");
    return JXB_ERR_ARG;
  }
  // Register budget by launch size: up to 256 threads, 512, 1024; the wide float
  // kernels (two CTAs per SM, 128 registers) for single-problem launches of up to 256.
  const bool multi = a.multi != nullptr;
  SimKernel kern = nullptr;
  if (a.wide && threads <= 256 && !multi) kern = pick_kernel<T>(backward, threads, gm, false, true);
  if (!kern) kern = pick_kernel<T>(backward, threads, gm, multi, false);
  if (!kern) {
    snprintf(g_err, sizeof(g_err), "no kernel instantiation for this launch shape");
    return JXB_ERR_ARG;
  }
  cudaError_t e = grant_smem((const void*)kern, smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute", e);
    return JXB_ERR_LAUNCH;
  }
  kern<<<a.n_items, threads, smem, stream>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err(backward ? "sim_backward_kernel" : "sim_forward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

static int check_sim_args(const JxbSimArgs* a, bool backward) {
  if (!a) return JXB_ERR_ARG;
  if (a->dtype != JXB_F32 && a->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (a->n_items <= 0) return JXB_OK;
  if (!a->node_class || !a->soff || !a->poff || !a->a_low || !a->a_up || !a->gsum || !a->cm ||
      !a->cls_ptr || !a->cls_comp || !a->entries || !a->pbase || !a->pcol || !a->pscale ||
      !a->blocks || !a->items || !a->chain_top || !a->chain_len || !a->chain_ptop ||
      !a->chain_cptr || !a->level_ptr || !a->stim_ptr || !a->state || !a->area ||
      !a->parent || !a->kid_ptr || !a->kid || !a->gk || !a->gbase) {
    snprintf(g_err, sizeof(g_err), "null pointer in JxbSimArgs");
    return JXB_ERR_ARG;
  }
  if (a->max_rows <= 0 || a->max_nodes <= 0 || a->max_nodes > 32767 || a->max_slots <= 0) {
    snprintf(g_err, sizeof(g_err), "bad block sizes (nodes per block must be 1..32767)");
    return JXB_ERR_ARG;
  }
  if (a->n_rec > 0 && (!a->rec_ptr || !a->rec_slot || !a->rec_col)) {
    snprintf(g_err, sizeof(g_err), "recordings without their index arrays");
    return JXB_ERR_ARG;
  }
  if (!backward && a->n_rec > 0 && !a->rec_out) {
    snprintf(g_err, sizeof(g_err), "recordings without output buffer");
    return JXB_ERR_ARG;
  }
  if (a->n_stim > 0 && (!a->stim || !a->stim_idx || a->stim_rows <= 0)) {
    snprintf(g_err, sizeof(g_err), "stimulus indices without stimulus");
    return JXB_ERR_ARG;
  }
  if (a->ckpt && !backward && a->ckpt_every <= 0) {
    snprintf(g_err, sizeof(g_err), "ckpt_every must be positive");
    return JXB_ERR_ARG;
  }
  if (a->clamp_ptr && (!a->clamp_slot || !a->clamp_col || !a->clamp || a->n_clamp <= 0 ||
                       (a->clamp_rows != 1 && a->clamp_rows < a->batch) ||
                       (a->mode == 0 && a->t0 + a->n_steps > a->clamp_steps))) {
    snprintf(g_err, sizeof(g_err),
             "clamps: index arrays, values of 1 or batch rows and at least t0 + n_steps time steps needed");
    return JXB_ERR_ARG;
  }
  if ((a->syn_lin == nullptr) != (a->syn_const == nullptr)) return JXB_ERR_ARG;
  if (a->syn_lin && a->n_steps != 1) {
    snprintf(g_err, sizeof(g_err), "synaptic terms require one step per launch");
    return JXB_ERR_ARG;
  }
  if (backward) {
    if (!a->ckpt || !a->traj || !a->traj_piv || !a->adj || !a->pgrad || a->mode != 0 ||
        a->n_steps <= 0) {
      snprintf(g_err, sizeof(g_err), "adjoint needs ckpt, traj, traj_piv, adj, pgrad and n_steps > 0");
      return JXB_ERR_ARG;
    }
  }
  return JXB_OK;
}

int check_sim_args_public(const JxbSimArgs* a, bool backward) { return check_sim_args(a, backward); }

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_sim_forward(const JxbSimArgs* a, void* stream) {
  int rc = check_sim_args(a, false);
  if (rc != JXB_OK || a->n_items <= 0) return rc;
  if (a->dtype == JXB_F32) return launch_sim<float>(*a, false, (cudaStream_t)stream);
  return launch_sim<double>(*a, false, (cudaStream_t)stream);
}

extern "C" int jxb_sim_backward(const JxbSimArgs* a, void* stream) {
  int rc = check_sim_args(a, true);
  if (rc != JXB_OK || a->n_items <= 0) return rc;
  if (a->dtype == JXB_F32) return launch_sim<float>(*a, true, (cudaStream_t)stream);
  return launch_sim<double>(*a, true, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------------
// Continuous batching: one launch over the work items of several problems.
// ---------------------------------------------------------------------------------
static size_t multi_pairs_offset(int n_reqs) { return (sizeof(JxbSimArgs) * (size_t)n_reqs + 255) / 256 * 256; }

extern "C" int64_t jxb_sim_multi_scratch_bytes(int n_reqs, int n_pairs) {
  if (n_reqs < 0 || n_pairs < 0) return -1;
  return (int64_t)(multi_pairs_offset(n_reqs) + sizeof(int32_t) * 2 * (size_t)n_pairs);
}

static int launch_multi(const JxbSimArgs* launch, const JxbSimArgs* reqs, int n_reqs, const int32_t* pairs,
                        int n_pairs, void* dev_scratch, int64_t scratch_bytes, void* stream, bool backward) {
  if (!launch || (n_reqs > 0 && !reqs) || (n_pairs > 0 && !pairs) || n_reqs < 0 || n_pairs < 0)
    return JXB_ERR_ARG;
  if (launch->dtype != JXB_F32 && launch->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (n_pairs == 0) return JXB_OK;
  if (!dev_scratch || ((uintptr_t)dev_scratch & 255) != 0 ||
      scratch_bytes < jxb_sim_multi_scratch_bytes(n_reqs, n_pairs)) {
    snprintf(g_err, sizeof(g_err), "multi launch: device scratch of %lld bytes (256-byte aligned) needed",
             (long long)jxb_sim_multi_scratch_bytes(n_reqs, n_pairs));
    return JXB_ERR_ARG;
  }
  const JxbSimArgs& L = *launch;
  if (L.max_rows <= 0 || L.max_nodes <= 0 || L.max_nodes > 32767 || L.max_slots <= 0) {
    snprintf(g_err, sizeof(g_err), "multi launch: bad block sizes");
    return JXB_ERR_ARG;
  }
  for (int r = 0; r < n_reqs; ++r) {
    const JxbSimArgs& q = reqs[r];
    if (q.dtype != L.dtype) return JXB_ERR_DTYPE;
    int rc = check_sim_args(&q, backward);
    if (rc != JXB_OK) return rc;
    if (q.max_rows > L.max_rows || q.max_nodes > L.max_nodes || q.max_slots > L.max_slots ||
        q.max_chains > L.max_chains || q.max_child > L.max_child || q.max_levels > L.max_levels ||
        q.max_pslots > L.max_pslots || q.n_entries > L.n_entries || q.n_classes > L.n_classes ||
        (backward && q.max_gslots > L.max_gslots)) {
      snprintf(g_err, sizeof(g_err), "multi launch: request %d exceeds the launch's block sizes", r);
      return JXB_ERR_ARG;
    }
  }
  for (int k = 0; k < n_pairs; ++k) {
    const int r = pairs[2 * k], it = pairs[2 * k + 1];
    if (r < 0 || r >= n_reqs || it < 0 || it >= reqs[r].n_items) {
      snprintf(g_err, sizeof(g_err), "multi launch: pair %d (request %d, item %d) out of range", k, r, it);
      return JXB_ERR_ARG;
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  char* dev = (char*)dev_scratch;
  cudaError_t e = cudaMemcpyAsync(dev, reqs, sizeof(JxbSimArgs) * (size_t)n_reqs, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dev + multi_pairs_offset(n_reqs), pairs, sizeof(int32_t) * 2 * (size_t)n_pairs,
                        cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) {
    set_err("cudaMemcpyAsync", e);
    return JXB_ERR_LAUNCH;
  }
  JxbSimArgs M = L;
  M.multi = (const JxbSimArgs*)dev;
  M.multi_items = (const int32_t*)(dev + multi_pairs_offset(n_reqs));
  M.n_items = n_pairs;
  if (M.dtype == JXB_F32) return launch_sim<float>(M, backward, st);
  return launch_sim<double>(M, backward, st);
}

extern "C" int jxb_sim_forward_multi(const JxbSimArgs* launch, const JxbSimArgs* reqs, int n_reqs,
                                     const int32_t* pairs, int n_pairs, void* dev_scratch,
                                     int64_t scratch_bytes, void* stream) {
  return launch_multi(launch, reqs, n_reqs, pairs, n_pairs, dev_scratch, scratch_bytes, stream, false);
}

extern "C" int jxb_sim_backward_multi(const JxbSimArgs* launch, const JxbSimArgs* reqs, int n_reqs,
                                      const int32_t* pairs, int n_pairs, void* dev_scratch,
                                      int64_t scratch_bytes, void* stream) {
  return launch_multi(launch, reqs, n_reqs, pairs, n_pairs, dev_scratch, scratch_bytes, stream, true);
}

extern "C" int64_t jxb_sim_smem_bytes(const JxbSimArgs* a, int backward) {
  if (!a) return -1;
  if (a->dtype == JXB_F32) return (int64_t)sim_smem_layout<float>(*a, backward != 0, nullptr, nullptr);
  return (int64_t)sim_smem_layout<double>(*a, backward != 0, nullptr, nullptr);
}

extern "C" const char* jxb_last_error(void) { return g_err; }
extern "C" int jxb_version(void) { return 1; }

// ---------------------------------------------------------------------------------
// Adjoint segment without caller-provided scratch.
//
// Some callers cannot allocate device memory while they run the simulation: a
// host program that hands this library fixed buffers from its own memory pool and
// forbids allocation during a training loop, or a plugin that is invoked from a
// framework step whose allocator must not be re-entered. For them the trajectory
// scratch of the adjoint (state before every step of the segment plus the step's
// pivots) lives in this fixed device array instead of caller buffers. Every GPU that
// loads the library holds the array until the process exits.
// ---------------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;

// Device address of the array per device, together with the context it was looked up
// in: a context created after cudaDeviceReset loads the array at a new address, so
// the set-up runs again for it. Guarded by a mutex (calls may come from several host
// threads).
struct NoAllocSlot {
  void* ctx;
  void* ptr;
};
NoAllocSlot g_noalloc_slot[kMaxDevices] = {};
std::mutex g_noalloc_mu;

typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn g_ctx_get_current = nullptr;
std::once_flag g_ctx_fn_once;

// The current context of the calling thread (driver entry point cuCtxGetCurrent,
// looked up once through the runtime; no link against libcuda).
void* current_context() {
  std::call_once(g_ctx_fn_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = (CtxGetCurrentFn)fn;
  });
  void* ctx = nullptr;
  if (g_ctx_get_current) g_ctx_get_current(&ctx);
  return ctx;
}

// The array's device address on the current device (looked up on the first call in
// the device's current context).
cudaError_t noalloc_scratch(int dev, void** out) {
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& s = g_noalloc_slot[dev];
  if (!s.ptr || s.ctx != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    s.ptr = p;
    s.ctx = ctx;
  }
  *out = s.ptr;
  return cudaSuccess;
}

}  // namespace

extern "C" int jxb_sim_backward_noalloc(const JxbSimArgs* a, void* stream) {
  if (!a) return JXB_ERR_ARG;
  if (a->dtype != JXB_F32 && a->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (a->n_items <= 0) return JXB_OK;
  if (a->n_steps <= 0 || a->batch <= 0 || a->n_slots <= 0 || a->n_nodes <= 0) {
    snprintf(jxb::g_err, sizeof(jxb::g_err), "jxb_sim_backward_noalloc: bad sizes");
    return JXB_ERR_ARG;
  }
  const size_t item = a->dtype == JXB_F32 ? sizeof(float) : sizeof(double);
  const size_t traj_bytes = (size_t)a->n_steps * a->batch * a->n_slots * item;
  const size_t piv_off = (traj_bytes + 255) / 256 * 256;
  const size_t need = piv_off + (size_t)a->n_steps * a->batch * a->n_nodes * item;
  if (need > kNoAllocScratchBytes) {
    snprintf(jxb::g_err, sizeof(jxb::g_err),
             "jxb_sim_backward_noalloc: segment needs %zu bytes of scratch, the fixed "
             "array holds %zu (use fewer steps per segment or jxb_sim_backward)",
             need, kNoAllocScratchBytes);
    return JXB_ERR_TOO_LARGE;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    jxb::set_err("cudaGetDevice", e);
    return JXB_ERR_LAUNCH;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    snprintf(jxb::g_err, sizeof(jxb::g_err),
             "jxb_sim_backward_noalloc: device %d is beyond the %d devices the library tracks", dev,
             kMaxDevices);
    return JXB_ERR_ARG;
  }
  // Set-up on the first call per device and context (the device must be current):
  // the device address of the array. That call should come before any stream capture.
  void* scratch = nullptr;
  e = noalloc_scratch(dev, &scratch);
  if (e != cudaSuccess) {
    jxb::set_err("cudaGetSymbolAddress", e);
    return JXB_ERR_LAUNCH;
  }
  // The caller's trajectory pointers are ignored; the rest is checked and launched
  // as by jxb_sim_backward.
  JxbSimArgs b = *a;
  b.traj_stored = 0;  // the segment is recomputed into the library's array
  b.traj = scratch;
  b.traj_piv = (unsigned char*)scratch + piv_off;
  const int rc = jxb::check_sim_args(&b, true);
  if (rc != JXB_OK) return rc;
  if (b.dtype == JXB_F32) return jxb::launch_sim<float>(b, true, (cudaStream_t)stream);
  return jxb::launch_sim<double>(b, true, (cudaStream_t)stream);
}
