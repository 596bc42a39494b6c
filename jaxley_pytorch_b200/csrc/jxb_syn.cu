// Fixed in-degree synapse step (KineticSynapse, SigmoidRateSynapse) in the regular
// layout: E = T * k synapses ordered by postsynaptic target, k per target
// (jaxley-pytorch kernels/synapse_step.py, modules/network.py:381-478).
//
// Both passes run one CTA per target with one thread per synapse of the target
// (warps over chunks of 32 synapses, up to 1024 synapses per target). A thread keeps
// its synapse's parameters, area and presynaptic index in registers and walks the
// batch rows in blocks of kRowBlock rows, whose loads (state, presynaptic and target
// voltages) are independent and issued together. Sums over a target's synapses (the
// slope and offset of the forward, the target-voltage gradient of the backward) are
// warp reductions followed by a fixed-order sum over the CTA's warps in shared
// memory. The backward's parameter gradients are summed over the rows in the
// synapse's own thread (no cross-CTA reduction); its presynaptic voltage gradients
// go to an (E, batch) buffer, kRowBlock consecutive rows per thread, which a second
// kernel sums per presynaptic node through the transposed index. No atomics,
// deterministic. float: fast reciprocal / division / exp (jxb_math.cuh); float64
// stays exact.
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

constexpr int kRowBlock = 8;  // batch rows per register block
constexpr int kMaxWarps = 32;  // up to 1024 synapses per target

// Sums over the CTA's synapses of NV values per row of a block (lane sums, then the
// warps in a fixed order); thread r (r < nr) receives the sums of row r in out[].
// `red` holds NV x kMaxWarps x kRowBlock values.
template <typename T, int NV>
__device__ __forceinline__ void block_row_sums(T (&v)[NV][kRowBlock], int nr, T* red, T (&out)[NV]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int r = 0; r < kRowBlock; ++r) v[i][r] = warp_sum(v[i][r]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i)
#pragma unroll
      for (int r = 0; r < kRowBlock; ++r) red[(i * kMaxWarps + warp) * kRowBlock + r] = v[i][r];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    out[i] = T(0);
    if ((int)threadIdx.x < nr)
      for (int w = 0; w < nw; ++w) out[i] += red[(i * kMaxWarps + w) * kRowBlock + threadIdx.x];
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(1024) syn_forward_kernel(JxbSynArgs a, SynP<T> P) {
  __shared__ T red[2 * kMaxWarps * kRowBlock];
  const int tgt = blockIdx.x;
  const int kk = threadIdx.x;
  const bool act = kk < a.k;
  const int nt = a.n_syn / a.k;
  const int64_t e = (int64_t)tgt * a.k + (act ? kk : 0);
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  const int node = a.targets_are_nodes ? tgt : a.targets[tgt];
  const int pre = a.pre[e];
  const T gs = P.p[0][e];
  const T ar = ((const T*)a.area)[e];
  const T q1 = P.p[1][e], q2 = P.p[2][e];
  const T q3 = a.model == 0 ? P.p[3][e] : T(0), q4 = a.model == 0 ? P.p[4][e] : T(0),
          q5 = a.model == 0 ? P.p[5][e] : T(1);
  for (int b0 = 0; b0 < a.batch; b0 += kRowBlock) {
    const int nr = min(kRowBlock, a.batch - b0);
    T sums[2][kRowBlock];  // slope and offset of every row
#pragma unroll
    for (int r = 0; r < kRowBlock; ++r) {
      sums[0][r] = sums[1][r] = T(0);
      if (!act || r >= nr) continue;
      const int64_t b = b0 + r;
      const T* v = (const T*)a.v + b * a.n_nodes;
      const T vp = v[node];
      const T vpre = v[pre];
      T i0, i1;
      if (a.model == 0) {  // synapses/kinetic.py:37-63 (e_syn, alpha, beta, v_th, delta)
        const T s = ((const T*)a.s)[b * a.n_syn + e];
        const T tr = sigm(qdiv<T>(vpre - q4, q5));
        const T aa = q2 * tr;
        const T rate = aa + q3;
        const T s_inf = qdiv<T>(aa, rate);
        const T s_new = s_inf + (s - s_inf) * ex(-dt * rate);
        ((T*)a.s_new)[b * a.n_syn + e] = s_new;
        i0 = gs * s_new * (vp - q1);
        i1 = gs * s_new * ((vp + diff) - q1);
      } else {  // synapses/sigmoid_rate.py:43-50 (x_offset, slope)
        i0 = -gs * sigm((vpre - q1) * q2);
        i1 = -gs * sigm(((vpre + diff) - q1) * q2);
      }
      const T d0 = qdiv<T>(i0, ar) * T(100000.0);
      const T d1 = qdiv<T>(i1, ar) * T(100000.0);
      const T vt = qdiv<T>(d1 - d0, diff);
      sums[0][r] = vt;
      sums[1][r] = d0 - vt * vp;
      if (a.store_current) ((T*)a.current)[b * a.n_syn + e] = i0;
    }
    T tot[2];
    block_row_sums<T, 2>(sums, nr, red, tot);
    if ((int)threadIdx.x < nr) {
      ((T*)a.lin)[(int64_t)(b0 + threadIdx.x) * nt + tgt] = tot[0];
      ((T*)a.cst)[(int64_t)(b0 + threadIdx.x) * nt + tgt] = tot[1];
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(1024) syn_backward_kernel(JxbSynArgs a, SynP<T> P) {
  __shared__ T red[kMaxWarps * kRowBlock];
  const int tgt = blockIdx.x;
  const int kk = threadIdx.x;
  const bool act = kk < a.k;
  const int nt = a.n_syn / a.k;
  const int64_t e = (int64_t)tgt * a.k + (act ? kk : 0);
  const T* sc = (const T*)a.scalars;
  const T dt = sc[0], diff = sc[1];
  const int node = a.targets_are_nodes ? tgt : a.targets[tgt];
  const int pre = a.pre[e];
  const T gs = P.p[0][e];
  const T ar = ((const T*)a.area)[e];
  const T q1 = P.p[1][e], q2 = P.p[2][e];
  const T q3 = a.model == 0 ? P.p[3][e] : T(0), q4 = a.model == 0 ? P.p[4][e] : T(0),
          q5 = a.model == 0 ? P.p[5][e] : T(1);
  T gp[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};  // parameter gradients over the rows
  T* g_pre = (T*)a.g_pre;
  for (int b0 = 0; b0 < a.batch; b0 += kRowBlock) {
    const int nr = min(kRowBlock, a.batch - b0);
    T gvp[1][kRowBlock];
#pragma unroll
    for (int r = 0; r < kRowBlock; ++r) {
      gvp[0][r] = T(0);
      if (!act || r >= nr) continue;
      const int64_t b = b0 + r;
      const T* v = (const T*)a.v + b * a.n_nodes;
      const T vp = v[node];
      const T vpre = v[pre];
      const T glin = ((const T*)a.g_lin)[b * nt + tgt];
      const T gconst = ((const T*)a.g_const)[b * nt + tgt];
      // Forward quantities (kernels/synapse_step.py:225-255).
      T i0, i1, w0 = T(0), w1 = T(0), s = T(0), s_new = T(0), tr = T(0), rate = T(1), s_inf = T(0),
               decay = T(0), x = T(0), u0 = T(0), u1 = T(0), sig0 = T(0), sig1 = T(0);
      if (a.model == 0) {
        s = ((const T*)a.s)[b * a.n_syn + e];
        x = qdiv<T>(vpre - q4, q5);
        tr = sigm(x);
        const T aa = q2 * tr;
        rate = aa + q3;
        s_inf = qdiv<T>(aa, rate);
        decay = ex(-dt * rate);
        s_new = s_inf + (s - s_inf) * decay;
        w0 = vp - q1;
        w1 = (vp + diff) - q1;
        i0 = gs * s_new * w0;
        i1 = gs * s_new * w1;
      } else {
        u0 = vpre - q1;
        u1 = (vpre + diff) - q1;
        sig0 = sigm(u0 * q2);
        sig1 = sigm(u1 * q2);
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
        const T g_x = g_a * q2 * tr * (T(1) - tr);
        g_vpre = qdiv<T>(g_x, q5);
        ((T*)a.g_s)[b * a.n_syn + e] = g_sn * decay;
        gp[0] += s_new * g_w;
        gp[1] += -gs * s_new * (g_i0 + g_i1);
        gp[2] += g_a * tr;
        gp[3] += g_rate;
        gp[4] += -g_vpre;
        gp[5] += -g_vpre * x;
      } else {
        const T g_z0 = -gs * g_i0 * sig0 * (T(1) - sig0);
        const T g_z1 = -gs * g_i1 * sig1 * (T(1) - sig1);
        g_vpre = (g_z0 + g_z1) * q2;
        gp[0] += -(g_i0 * sig0 + g_i1 * sig1);
        gp[1] += -g_vpre;
        gp[2] += g_z0 * u0 + g_z1 * u1;
      }
      gvp[0][r] = g_vp;
      g_pre[e * a.batch + b] = g_vpre;
    }
    T tot[1];
    block_row_sums<T, 1>(gvp, nr, red, tot);
    const T g = tot[0];
    // The target-voltage gradient of row b0 + threadIdx.x: added to g_v here when
    // accumulating (this CTA owns the (row, target) pair), else by syn_post_kernel.
    if ((int)threadIdx.x < nr) {
      const int64_t b = b0 + threadIdx.x;
      if (a.accumulate) ((T*)a.g_v)[b * a.n_nodes + node] += g;
      else ((T*)a.g_post)[b * nt + tgt] = g;
    }
  }
  if (!act) return;
  const int np = a.model == 0 ? 6 : 3;
  int row = 0;
  for (int q = 0; q < np; ++q) {
    if (!(a.need & (1 << q))) continue;
    T& out = ((T*)a.g_params)[(int64_t)row * a.n_syn + e];
    out = a.accumulate ? out + gp[q] : gp[q];
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

// Threads per CTA: one per synapse of a target, rounded up to whole warps.
inline int syn_threads(int k) { return 32 * ((k + 31) / 32); }

template <typename T>
int fwd(const JxbSynArgs& a, cudaStream_t st) {
  SynP<T> P;
  for (int q = 0; q < 6; ++q) P.p[q] = (const T*)a.p[q];
  const int nt = a.n_syn / a.k;
  syn_forward_kernel<T><<<nt, syn_threads(a.k), 0, st>>>(a, P);
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
  syn_backward_kernel<T><<<nt, syn_threads(a.k), 0, st>>>(a, P);
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
  if (a->k > 32 * kMaxWarps) {
    snprintf(g_err, sizeof(g_err), "synapse step: %d synapses per target exceed %d", a->k, 32 * kMaxWarps);
    return JXB_ERR_TOO_LARGE;
  }
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
