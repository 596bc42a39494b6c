// Fixed in-degree synapse step (KineticSynapse, SigmoidRateSynapse) in the regular
// layout: E = T * k synapses ordered by postsynaptic target, k per target
// (jaxley-pytorch kernels/synapse_step.py, modules/network.py:381-478).
//
// forward:  one warp per target looping over the batch rows; lanes stride over the
//           target's k synapses (coalesced state reads, gathered presynaptic
//           voltages, parameters reused from L1 across the rows), the slope and
//           offset sums over k are warp reductions.
// backward: one CTA per target, warps over batch rows, lanes over synapses. The
//           parameter gradients (summed over the batch) are reduced across warps in
//           shared memory in a fixed order; the presynaptic voltage gradients of the
//           CTA's synapses are staged in shared memory and written to an (E, batch)
//           buffer row by row (coalesced), which a second kernel sums per
//           presynaptic node through the transposed index. No atomics, deterministic.
// float: fast reciprocal / division / exp (jxb_math.cuh); float64 stays exact.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "jxb.h"
#include "jxb_math.cuh"

namespace jxb {
extern thread_local char g_err[512];
void set_err(const char* what, cudaError_t e);
}  // namespace jxb

namespace {

using namespace jxb;

template <typename T> __device__ __forceinline__ T qdiv(T x, T y) { return jxb::fdiv(x, y); }
template <typename T> __device__ __forceinline__ T sigm(T x) { return jxb::rcp(T(1) + ex(-x)); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
struct SynP {
  const T* p[6];
};

template <typename T>
__global__ void syn_forward_kernel(JxbSynArgs a, SynP<T> P) {
  const int tgt = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nt = a.n_syn / a.k;
  if (tgt >= nt) return;
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  const int node = a.targets_are_nodes ? tgt : a.targets[tgt];
  const T* area = (const T*)a.area;
  for (int64_t b = 0; b < a.batch; ++b) {
    const T* v = (const T*)a.v + b * a.n_nodes;
    const T vp = v[node];
    T lin = T(0), cst = T(0);
    for (int kk = lane; kk < a.k; kk += 32) {
      const int e = tgt * a.k + kk;
      const T vpre = v[a.pre[e]];
      const T gs = P.p[0][e];
      T i0, i1;
      if (a.model == 0) {  // synapses/kinetic.py:37-63
        const T e_syn = P.p[1][e], alpha = P.p[2][e], beta = P.p[3][e], v_th = P.p[4][e],
                delta = P.p[5][e];
        const T s = ((const T*)a.s)[b * a.n_syn + e];
        const T tr = sigm(qdiv<T>(vpre - v_th, delta));
        const T aa = alpha * tr;
        const T rate = aa + beta;
        const T s_inf = qdiv<T>(aa, rate);
        const T s_new = s_inf + (s - s_inf) * ex(-dt * rate);
        ((T*)a.s_new)[b * a.n_syn + e] = s_new;
        i0 = gs * s_new * (vp - e_syn);
        i1 = gs * s_new * ((vp + diff) - e_syn);
      } else {  // synapses/sigmoid_rate.py:43-50
        const T x_off = P.p[1][e], slope = P.p[2][e];
        i0 = -gs * sigm((vpre - x_off) * slope);
        i1 = -gs * sigm(((vpre + diff) - x_off) * slope);
      }
      const T d0 = qdiv<T>(i0, area[e]) * T(100000.0);
      const T d1 = qdiv<T>(i1, area[e]) * T(100000.0);
      const T vt = qdiv<T>(d1 - d0, diff);
      lin += vt;
      cst += d0 - vt * vp;
      if (a.store_current) ((T*)a.current)[b * a.n_syn + e] = i0;
    }
    lin = warp_sum(lin);
    cst = warp_sum(cst);
    if (lane == 0) {
      ((T*)a.lin)[b * nt + tgt] = lin;
      ((T*)a.cst)[b * nt + tgt] = cst;
    }
  }
}

constexpr int kBwdWarps = 4;
constexpr int kStageBytes = 64 * 1024;  // largest staged (k, batch) tile of presynaptic gradients

template <typename T>
__global__ void syn_backward_kernel(JxbSynArgs a, SynP<T> P) {
  // red[warp][param][kk]: every warp (batch slice) accumulates its own parameter
  // gradients; summed over the warps in a fixed order at the end.
  extern __shared__ __align__(16) char smem_raw[];
  T* red = (T*)smem_raw;
  const int tgt = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nt = a.n_syn / a.k;
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  const int node = a.targets_are_nodes ? tgt : a.targets[tgt];
  const T* area = (const T*)a.area;
  const int np = a.model == 0 ? 6 : 3;
  T* g_pre = (T*)a.g_pre;
  T* myred = red + (size_t)warp * 6 * a.k;
  // the CTA's presynaptic gradients, (k, batch), staged for coalesced stores
  T* stile = a.batch * a.k * (int)sizeof(T) <= kStageBytes ? red + (size_t)kBwdWarps * 6 * a.k : nullptr;
  for (int q = lane; q < 6 * a.k; q += 32) myred[q] = T(0);
  __syncwarp();
  for (int64_t b = warp; b < a.batch; b += kBwdWarps) {
    const T* v = (const T*)a.v + b * a.n_nodes;
    const T vp = v[node];
    const T glin = ((const T*)a.g_lin)[b * nt + tgt];
    const T gconst = ((const T*)a.g_const)[b * nt + tgt];
    T gvp_sum = T(0);
    for (int kk = lane; kk < a.k; kk += 32) {
      T* gq = myred + kk;  // gradient of parameter q at gq[q * k]
      const int e = tgt * a.k + kk;
      const T vpre = v[a.pre[e]];
      const T gs = P.p[0][e];
      const T ar = area[e];
      // Forward quantities (kernels/synapse_step.py:225-255).
      T i0, i1, w0 = T(0), w1 = T(0), s = T(0), s_new = T(0), tr = T(0), rate = T(1),
               s_inf = T(0), decay = T(0), x = T(0), u0 = T(0), u1 = T(0), sig0 = T(0),
               sig1 = T(0), alpha = T(0), delta = T(1), slope = T(0);
      if (a.model == 0) {
        const T e_syn = P.p[1][e], beta = P.p[3][e], v_th = P.p[4][e];
        alpha = P.p[2][e];
        delta = P.p[5][e];
        s = ((const T*)a.s)[b * a.n_syn + e];
        x = qdiv<T>(vpre - v_th, delta);
        tr = sigm(x);
        const T aa = alpha * tr;
        rate = aa + beta;
        s_inf = qdiv<T>(aa, rate);
        decay = ex(-dt * rate);
        s_new = s_inf + (s - s_inf) * decay;
        w0 = vp - e_syn;
        w1 = (vp + diff) - e_syn;
        i0 = gs * s_new * w0;
        i1 = gs * s_new * w1;
      } else {
        const T x_off = P.p[1][e];
        slope = P.p[2][e];
        u0 = vpre - x_off;
        u1 = (vpre + diff) - x_off;
        sig0 = sigm(u0 * slope);
        sig1 = sigm(u1 * slope);
        i0 = -gs * sig0;
        i1 = -gs * sig1;
      }
      const T d0 = qdiv<T>(i0, ar) * T(100000.0);
      const T d1 = qdiv<T>(i1, ar) * T(100000.0);
      const T vt = qdiv<T>(d1 - d0, diff);
      // Backward (kernels/synapse_step.py:256-305).
      const T g_vt = glin - gconst * vp;
      T g_vp = -gconst * vt;
      const T g_d1 = qdiv<T>(g_vt, diff);
      const T g_d0 = gconst - g_d1;
      T g_i0 = qdiv<T>(g_d0 * T(100000.0), ar);
      const T g_i1 = qdiv<T>(g_d1 * T(100000.0), ar);
      if (a.g_current) g_i0 += ((const T*)a.g_current)[b * a.n_syn + e];
      T g_vpre;
      if (a.model == 0) {
        const T g_w = g_i0 * w0 + g_i1 * w1;
        T g_sn = gs * g_w;
        if (a.g_s_new) g_sn += ((const T*)a.g_s_new)[b * a.n_syn + e];
        g_vp += gs * s_new * (g_i0 + g_i1);
        const T g_sinf = g_sn * (T(1) - decay);
        const T g_rate = -dt * decay * g_sn * (s - s_inf) - qdiv<T>(g_sinf * s_inf, rate);
        const T g_a = qdiv<T>(g_sinf, rate) + g_rate;
        const T g_x = g_a * alpha * tr * (T(1) - tr);
        g_vpre = qdiv<T>(g_x, delta);
        ((T*)a.g_s)[b * a.n_syn + e] = g_sn * decay;
        gq[0] += s_new * g_w;
        gq[a.k] += -gs * s_new * (g_i0 + g_i1);
        gq[2 * a.k] += g_a * tr;
        gq[3 * a.k] += g_rate;
        gq[4 * a.k] += -g_vpre;
        gq[5 * a.k] += -g_vpre * x;
      } else {
        const T g_z0 = -gs * g_i0 * sig0 * (T(1) - sig0);
        const T g_z1 = -gs * g_i1 * sig1 * (T(1) - sig1);
        g_vpre = (g_z0 + g_z1) * slope;
        gq[0] += -(g_i0 * sig0 + g_i1 * sig1);
        gq[a.k] += -g_vpre;
        gq[2 * a.k] += g_z0 * u0 + g_z1 * u1;
      }
      gvp_sum += g_vp;
      if (stile) stile[(size_t)kk * a.batch + b] = g_vpre;
      else g_pre[(int64_t)e * a.batch + b] = g_vpre;
    }
    gvp_sum = warp_sum(gvp_sum);
    // The postsynaptic voltage gradient of this row: added to g_v at the target here
    // when accumulating (one warp owns the (row, target) pair), else by
    // syn_post_kernel.
    if (lane == 0) {
      if (a.accumulate) ((T*)a.g_v)[b * a.n_nodes + node] += gvp_sum;
      else ((T*)a.g_post)[b * nt + tgt] = gvp_sum;
    }
  }
  // Sum the parameter gradients over the warps (batch slices), fixed order.
  __syncthreads();
  if (stile) {
    const int n = a.k * a.batch;
    T* dst = g_pre + (int64_t)tgt * a.k * a.batch;  // rows e = tgt * k + kk are consecutive
    for (int q = threadIdx.x; q < n; q += blockDim.x) dst[q] = stile[q];
  }
  int row = 0;
  for (int q = 0; q < np; ++q) {
    if (!(a.need & (1 << q))) continue;
    for (int kk = threadIdx.x; kk < a.k; kk += blockDim.x) {
      T acc = T(0);
      for (int w = 0; w < kBwdWarps; ++w) acc += red[((size_t)w * 6 + q) * a.k + kk];
      T& out = ((T*)a.g_params)[(int64_t)row * a.n_syn + tgt * a.k + kk];
      out = a.accumulate ? out + acc : acc;
    }
    ++row;
  }
}

// g_v[b, pre_nodes[j]] = sum over the synapses of node j of g_pre[e, b]; then the
// postsynaptic terms g_post[b, t] are added at the targets.
template <typename T>
__global__ void syn_presum_kernel(JxbSynArgs a) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)a.n_pre_nodes * a.batch) return;
  const int j = idx / a.batch;
  const int64_t b = idx % a.batch;
  const T* g_pre = (const T*)a.g_pre;
  T acc = T(0);
  for (int q = 0; q < a.inv_width; ++q) {
    const int e = a.inv[(int64_t)j * a.inv_width + q];
    if (e >= 0) acc += g_pre[(int64_t)e * a.batch + b];
  }
  T& out = ((T*)a.g_v)[b * a.n_nodes + a.pre_nodes[j]];
  out = a.accumulate ? out + acc : acc;
}

template <typename T>
__global__ void syn_post_kernel(JxbSynArgs a) {
  const int nt = a.n_syn / a.k;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nt * a.batch) return;
  const int t = idx % nt;
  const int64_t b = idx / nt;
  const int node = a.targets_are_nodes ? t : a.targets[t];
  ((T*)a.g_v)[b * a.n_nodes + node] += ((const T*)a.g_post)[b * nt + t];
}

template <typename T>
int fwd(const JxbSynArgs& a, cudaStream_t st) {
  SynP<T> P;
  for (int q = 0; q < 6; ++q) P.p[q] = (const T*)a.p[q];
  const int nt = a.n_syn / a.k;
  const int64_t warps = (int64_t)nt;  // one warp per target, looping over the rows
  const int threads = 128;
  syn_forward_kernel<T><<<(unsigned)((warps * 32 + threads - 1) / threads), threads, 0, st>>>(a, P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("syn_forward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

template <typename T>
int bwd(const JxbSynArgs& a, cudaStream_t st) {
  SynP<T> P;
  for (int q = 0; q < 6; ++q) P.p[q] = (const T*)a.p[q];
  const int nt = a.n_syn / a.k;
  cudaError_t e = cudaSuccess;
  if (!a.accumulate) {  // the op's g_v: zero where neither sum writes
    e = cudaMemsetAsync(a.g_v, 0, sizeof(T) * (size_t)a.batch * a.n_nodes, st);
    if (e != cudaSuccess) {
      set_err("cudaMemsetAsync", e);
      return JXB_ERR_LAUNCH;
    }
  }
  const size_t stage = sizeof(T) * (size_t)a.k * a.batch;
  const size_t smem = sizeof(T) * (size_t)kBwdWarps * 6 * a.k + (stage <= (size_t)kStageBytes ? stage : 0);
  if (smem > 227 * 1024) {
    snprintf(g_err, sizeof(g_err), "synapse backward: %d synapses per target exceed shared memory", a.k);
    return JXB_ERR_TOO_LARGE;
  }
  e = cudaFuncSetAttribute(syn_backward_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute", e);
    return JXB_ERR_LAUNCH;
  }
  syn_backward_kernel<T><<<nt, 32 * kBwdWarps, smem, st>>>(a, P);
  const int threads = 256;
  const int64_t n1 = (int64_t)a.n_pre_nodes * a.batch;
  if (n1 > 0) syn_presum_kernel<T><<<(unsigned)((n1 + threads - 1) / threads), threads, 0, st>>>(a);
  const int64_t n2 = (int64_t)nt * a.batch;
  if (!a.accumulate) syn_post_kernel<T><<<(unsigned)((n2 + threads - 1) / threads), threads, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("syn_backward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

int check(const JxbSynArgs* a, bool backward) {
  if (!a || a->k <= 0 || a->n_syn % a->k != 0 || a->batch <= 0 || !a->v || !a->pre ||
      !a->area || !a->scalars || !a->p[0])
    return JXB_ERR_ARG;
  if (a->model != 0 && a->model != 1) return JXB_ERR_ARG;
  if (a->model == 0 && (!a->s || !a->p[5])) return JXB_ERR_ARG;
  if (!a->targets_are_nodes && !a->targets) return JXB_ERR_ARG;
  if (a->dtype != JXB_F32 && a->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (!backward) {
    if (!a->lin || !a->cst) return JXB_ERR_ARG;
    if (a->model == 0 && !a->s_new) return JXB_ERR_ARG;
    if (a->store_current && !a->current) return JXB_ERR_ARG;
  } else {
    if ((!a->accumulate && !a->g_post) || !a->g_lin || !a->g_const || !a->g_v || !a->g_pre || !a->inv ||
        !a->pre_nodes)
      return JXB_ERR_ARG;
    if (a->model == 0 && !a->g_s) return JXB_ERR_ARG;
    if (a->need && !a->g_params) return JXB_ERR_ARG;
  }
  return JXB_OK;
}

}  // namespace

extern "C" int jxb_synapse_forward(const JxbSynArgs* a, void* stream) {
  int rc = check(a, false);
  if (rc) return rc;
  return a->dtype == JXB_F32 ? fwd<float>(*a, (cudaStream_t)stream) : fwd<double>(*a, (cudaStream_t)stream);
}

extern "C" int jxb_synapse_backward(const JxbSynArgs* a, void* stream) {
  int rc = check(a, true);
  if (rc) return rc;
  return a->dtype == JXB_F32 ? bwd<float>(*a, (cudaStream_t)stream) : bwd<double>(*a, (cudaStream_t)stream);
}
