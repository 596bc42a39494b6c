// Fused bwd_euler + DHS simulation kernels.
//
// One CTA owns one work item: a block of whole trees (cells) and a few batch rows.
// The rows' state vectors live in shared memory for the whole segment of steps; the
// per-step work is
//   1. channels, node-parallel: gate updates in insertion order, linearised currents
//      (modules/base.py:3402-3542), stimulus (:3234-3242), assembly of the diagonal
//      and right-hand side of the implicit system (solver_voltage.py:250-291);
//   2. the Hines solve of every tree (solver_voltage.py:78-108), organised by chains
//      (a node and its only child share a chain): one thread eliminates a whole
//      chain bottom-up in registers, chains of one level run in parallel and levels
//      are separated by a barrier; back-substitution runs the levels top-down.
// Recordings, checkpoints and the trajectory for the adjoint are written from the
// resident state.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "jxb.h"
#include "jxb_node.cuh"

namespace jxb {

thread_local char g_err[512] = "";

void set_err(const char* what, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", what, e == cudaSuccess ? "ok" : cudaGetErrorString(e));
}

template <typename T>
struct SimSmem {
  T* st;    // rows * n_slots
  T* D;     // rows * n_nodes
  T* S;     // rows * n_nodes
  T* al;    // n_nodes: -dt * a_low
  T* au;    // n_nodes: -dt * a_up
  T* dg;    // n_nodes: is_comp + dt * gsum
  T* cm;    // n_nodes
  T* adj;   // rows * n_slots (adjoint only)
  T* X1;    // rows * n_nodes (adjoint only)
  ChanEntry* ents;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

template <typename T>
__host__ __device__ inline size_t sim_smem_layout(const JxbSimArgs& a, bool backward, SimSmem<T>* out,
                                                  char* base) {
  size_t rows = a.max_rows, nn = a.max_nodes, ns = a.max_slots;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes, 16);
    return o;
  };
  size_t o_st = take(sizeof(T) * rows * ns);
  size_t o_D = take(sizeof(T) * rows * nn);
  size_t o_S = take(sizeof(T) * rows * nn);
  size_t o_al = take(sizeof(T) * nn);
  size_t o_au = take(sizeof(T) * nn);
  size_t o_dg = take(sizeof(T) * nn);
  size_t o_cm = take(sizeof(T) * nn);
  size_t o_adj = backward ? take(sizeof(T) * rows * ns) : 0;
  size_t o_X1 = backward ? take(sizeof(T) * rows * nn) : 0;
  size_t o_e = take(sizeof(ChanEntry) * (size_t)a.n_entries);
  if (out) {
    out->st = (T*)(base + o_st);
    out->D = (T*)(base + o_D);
    out->S = (T*)(base + o_S);
    out->al = (T*)(base + o_al);
    out->au = (T*)(base + o_au);
    out->dg = (T*)(base + o_dg);
    out->cm = (T*)(base + o_cm);
    out->adj = backward ? (T*)(base + o_adj) : nullptr;
    out->X1 = backward ? (T*)(base + o_X1) : nullptr;
    out->ents = (ChanEntry*)(base + o_e);
  }
  return off;
}

// Loads the block's shared topology and the rows' states into shared memory.
template <typename T>
__device__ void load_item(const JxbSimArgs& a, const JxbBlock& blk, int row0, int rows,
                          const SimSmem<T>& sm, T dt) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = blk.n_nodes, ns = blk.n_slots;
  const T* gl = (const T*)a.a_low;
  const T* gu = (const T*)a.a_up;
  const T* gs = (const T*)a.gsum;
  const T* cmv = (const T*)a.cm;
  for (int j = tid; j < nn; j += NT) {
    int i = blk.node0 + j;
    sm.al[j] = -(dt * gl[i]);
    sm.au[j] = -(dt * gu[i]);
    T comp = a.cls_comp[a.node_class[i]] ? T(1) : T(0);
    sm.dg[j] = comp + dt * gs[i];
    sm.cm[j] = cmv[i];
  }
  const short* src = (const short*)a.entries;
  short* dst = (short*)sm.ents;
  int nshort = a.n_entries * (int)(sizeof(ChanEntry) / sizeof(short));
  for (int q = tid; q < nshort; q += NT) dst[q] = src[q];
  const T* state = (const T*)a.state;
  for (int r = 0; r < rows; ++r) {
    const T* g = state + (size_t)(row0 + r) * a.n_slots + blk.slot0;
    T* s = sm.st + (size_t)r * ns;
    for (int q = tid; q < ns; q += NT) s[q] = g[q];
  }
}

// Chain elimination (leaves first) and back-substitution of every tree of the block
// for all rows. `al`/`au` are the matrix entries A[i, parent] / A[parent, i]; the
// adjoint passes them swapped to solve with the transposed matrix. On return `S`
// holds the solution.
template <typename T>
__device__ void block_solve(const JxbSimArgs& a, const JxbBlock& blk, int rows, T* D, T* S,
                            const T* al, const T* au) {
  const int tid = threadIdx.x, NT = blockDim.x;
  const int nn = blk.n_nodes, node0 = blk.node0;
  const int* lp = a.level_ptr + blk.level0;
  const int nlev = blk.n_levels;
  // Elimination, leaf chains first (solver_voltage.py:93-98).
  for (int h = 0; h < nlev; ++h) {
    int c0 = lp[h], nch = lp[h + 1] - c0;
    for (int w = tid; w < nch * rows; w += NT) {
      int c = blk.chain0 + c0 + w % nch;
      int r = w / nch;
      T* Dr = D + (size_t)r * nn;
      T* Sr = S + (size_t)r * nn;
      int top = a.chain_top[c] - node0;
      int bot = top + a.chain_len[c] - 1;
      T d = Dr[bot], s = Sr[bot];
      for (int k = a.chain_cptr[c]; k < a.chain_cptr[c + 1]; ++k) {
        int ct = a.chain_child[k] - node0;
        T f = au[ct] / Dr[ct];
        d -= al[ct] * f;
        s -= Sr[ct] * f;
      }
      Dr[bot] = d;
      Sr[bot] = s;
      for (int j = bot - 1; j >= top; --j) {
        T f = au[j + 1] / d;
        d = Dr[j] - al[j + 1] * f;
        s = Sr[j] - s * f;
        Dr[j] = d;
        Sr[j] = s;
      }
    }
    __syncthreads();
  }
  // Back-substitution, root chains first (solver_voltage.py:100-106).
  for (int h = nlev - 1; h >= 0; --h) {
    int c0 = lp[h], nch = lp[h + 1] - c0;
    for (int w = tid; w < nch * rows; w += NT) {
      int c = blk.chain0 + c0 + w % nch;
      int r = w / nch;
      T* Dr = D + (size_t)r * nn;
      T* Sr = S + (size_t)r * nn;
      int top = a.chain_top[c] - node0;
      int bot = top + a.chain_len[c] - 1;
      int pt = a.chain_ptop[c];
      T xp = pt >= 0 ? Sr[pt - node0] : T(0);
      for (int j = top; j <= bot; ++j) {
        T x = (Sr[j] - al[j] * xp) / Dr[j];
        Sr[j] = x;
        xp = x;
      }
    }
    __syncthreads();
  }
}

// Channel step of one node and row: updates the node's states and returns the
// linearised membrane terms (slope, offset) in uA/cm^2 (before the division by cm).
template <typename T>
__device__ __forceinline__ void node_forward(const JxbSimArgs& a, const SimSmem<T>& sm, int i,
                                             T* x, int b, T dt, int mode, T& lin, T& cst) {
  const int cls = a.node_class[i];
  const int e0 = a.cls_ptr[cls], e1 = a.cls_ptr[cls + 1];
  const int po = a.poff[i];
  Prm<T> P{(const T*)a.pbase + po, a.pcol + po, (const T*)a.pscale + (size_t)b * a.n_cols};
  const T v = x[0];
  if (mode == 0) {
    for (int q = e0; q < e1; ++q) {
      ChanEntry e = sm.ents[q];
      Prm<T> Pe{P.base + e.p[0], P.col + e.p[0], P.scale};
      channel_update<T>(e, x, Pe, v, dt);
    }
  } else if (mode == 2) {
    for (int q = e0; q < e1; ++q) channel_steady<T>(sm.ents[q], x, v);
    lin = cst = T(0);
    return;
  }
  for (int q = e0; q < e1; ++q) x[sm.ents[q].cur] = T(0);
  T slope = T(0), gge = T(0);
  for (int q = e0; q < e1; ++q) {
    ChanEntry e = sm.ents[q];
    Prm<T> Pe{P.base + e.p[0], P.col + e.p[0], P.scale};
    channel_current<T>(e, x, Pe, v, slope, gge);
  }
  lin = slope * T(1000.0);  // mA/cm^2 -> uA/cm^2, modules/base.py:3500-3502
  cst = gge * T(1000.0);
}

template <typename T>
__device__ __forceinline__ T stim_current(const JxbSimArgs& a, int i, int b, int t) {
  T acc = T(0);
  int q0 = a.stim_ptr[i], q1 = a.stim_ptr[i + 1];
  if (q0 == q1 || t >= a.stim_steps) return acc;
  const T* st = (const T*)a.stim + (size_t)t * a.stim_rows * a.n_stim +
                (size_t)(a.stim_rows == 1 ? 0 : b) * a.n_stim;
  const T area = ((const T*)a.area)[i];
  for (int q = q0; q < q1; ++q) acc += st[a.stim_idx[q]] / area * T(100000);
  return acc;
}

// Recordings of node i at time index t (integrate.py:53-84).
template <typename T>
__device__ __forceinline__ void record_node(const JxbSimArgs& a, int i, const T* x, int b, int t) {
  T* out = (T*)a.rec_out;
  for (int q = a.rec_ptr[i]; q < a.rec_ptr[i + 1]; ++q) {
    int sl = a.rec_slot[q];
    out[((size_t)t * a.batch + b) * a.n_rec + a.rec_col[q]] = sl >= 0 ? x[sl] : T(0);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) sim_forward_kernel(JxbSimArgs a) {
  extern __shared__ __align__(16) char smem_raw[];
  SimSmem<T> sm;
  sim_smem_layout<T>(a, false, &sm, smem_raw);
  const JxbItem item = a.items[blockIdx.x];
  const JxbBlock blk = a.blocks[item.block];
  const int rows = item.n_rows, row0 = item.row0;
  const int nn = blk.n_nodes, ns = blk.n_slots;
  const int tid = threadIdx.x, NT = blockDim.x;
  const T dt = T(a.dt);
  load_item<T>(a, blk, row0, rows, sm, dt);
  __syncthreads();

  const int total = nn * rows;
  const int nsteps = a.mode == 0 ? a.n_steps : 0;
  for (int step = 0; step <= nsteps; ++step) {
    const int t = a.t0 + step;
    for (int w = tid; w < total; w += NT) {
      const int r = w / nn, j = w % nn;
      const int i = blk.node0 + j;
      const int b = row0 + r;
      T* x = sm.st + (size_t)r * ns + (a.soff[i] - blk.slot0);
      const int nslot = a.soff[i + 1] - a.soff[i];
      if (step > 0) x[0] = sm.S[(size_t)r * nn + j];
      if (step > 0 && a.n_rec > 0) record_node<T>(a, i, x, b, t);
      if (step == nsteps) {
        if (a.mode != 0) {
          // Initial currents (mode 1, modules/base.py:2375-2383), after the steady
          // state of every channel (mode 2, modules/base.py:2419-2474).
          T lin, cst;
          if (a.mode == 2) node_forward<T>(a, sm, i, x, b, dt, 2, lin, cst);
          node_forward<T>(a, sm, i, x, b, dt, 1, lin, cst);
          if (a.n_rec > 0) record_node<T>(a, i, x, b, t);
        }
        T* g = (T*)a.state + (size_t)b * a.n_slots + a.soff[i];
        for (int q = 0; q < nslot; ++q) g[q] = x[q];
        continue;
      }
      if (a.traj) {
        T* g = (T*)a.traj + ((size_t)step * a.batch + b) * a.n_slots + a.soff[i];
        for (int q = 0; q < nslot; ++q) g[q] = x[q];
      }
      if (a.ckpt && ((t - a.ckpt_base) % a.ckpt_every) == 0) {
        size_t m = (size_t)((t - a.ckpt_base) / a.ckpt_every);
        T* g = (T*)a.ckpt + (m * a.batch + b) * a.n_slots + a.soff[i];
        for (int q = 0; q < nslot; ++q) g[q] = x[q];
      }
      const T v = x[0];
      T lin, cst;
      node_forward<T>(a, sm, i, x, b, dt, 0, lin, cst);
      T iext = stim_current<T>(a, i, b, t);
      if (a.syn_lin) {
        lin += ((const T*)a.syn_lin)[(size_t)b * a.n_nodes + i];
        cst += ((const T*)a.syn_const)[(size_t)b * a.n_nodes + i];
      }
      const T cmv = sm.cm[j];
      const T lin_t = lin / cmv;
      const T cst_t = (cst + iext) / cmv;
      const bool comp = a.cls_comp[a.node_class[i]] != 0;
      sm.D[(size_t)r * nn + j] = sm.dg[j] + dt * lin_t;
      sm.S[(size_t)r * nn + j] = comp ? v + dt * cst_t : T(0);
    }
    if (step == nsteps) break;
    __syncthreads();
    block_solve<T>(a, blk, rows, sm.D, sm.S, sm.al, sm.au);
  }
}

template <typename T>
int launch_forward(const JxbSimArgs& a, cudaStream_t stream) {
  size_t smem = sim_smem_layout<T>(a, false, nullptr, nullptr);
  if (smem > 227 * 1024) {
    snprintf(g_err, sizeof(g_err), "work item needs %zu bytes of shared memory", smem);
    return JXB_ERR_SMEM;
  }
  cudaError_t e = cudaFuncSetAttribute(sim_forward_kernel<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute", e);
    return JXB_ERR_LAUNCH;
  }
  sim_forward_kernel<T><<<a.n_items, 256, smem, stream>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("sim_forward_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

static int check_sim_args(const JxbSimArgs* a) {
  if (!a) return JXB_ERR_ARG;
  if (a->dtype != JXB_F32 && a->dtype != JXB_F64) return JXB_ERR_DTYPE;
  if (a->n_items <= 0) return JXB_OK;
  if (!a->node_class || !a->soff || !a->poff || !a->a_low || !a->a_up || !a->gsum || !a->cm ||
      !a->cls_ptr || !a->cls_comp || !a->entries || !a->pbase || !a->pcol || !a->pscale ||
      !a->blocks || !a->items || !a->chain_top || !a->chain_len || !a->chain_ptop ||
      !a->chain_cptr || !a->level_ptr || !a->stim_ptr || !a->state || !a->area) {
    snprintf(g_err, sizeof(g_err), "null pointer in JxbSimArgs");
    return JXB_ERR_ARG;
  }
  if (a->n_rec > 0 && (!a->rec_out || !a->rec_ptr || !a->rec_slot || !a->rec_col)) {
    snprintf(g_err, sizeof(g_err), "recordings without output buffer");
    return JXB_ERR_ARG;
  }
  if (a->n_stim > 0 && (!a->stim || !a->stim_idx || a->stim_rows <= 0)) {
    snprintf(g_err, sizeof(g_err), "stimulus indices without stimulus");
    return JXB_ERR_ARG;
  }
  if (a->ckpt && a->ckpt_every <= 0) {
    snprintf(g_err, sizeof(g_err), "ckpt_every must be positive");
    return JXB_ERR_ARG;
  }
  if ((a->syn_lin == nullptr) != (a->syn_const == nullptr)) return JXB_ERR_ARG;
  if (a->syn_lin && a->n_steps != 1) {
    snprintf(g_err, sizeof(g_err), "synaptic terms require one step per launch");
    return JXB_ERR_ARG;
  }
  return JXB_OK;
}

}  // namespace jxb

using namespace jxb;

extern "C" int jxb_sim_forward(const JxbSimArgs* a, void* stream) {
  int rc = check_sim_args(a);
  if (rc != JXB_OK || a->n_items <= 0) return rc;
  if (a->dtype == JXB_F32) return launch_forward<float>(*a, (cudaStream_t)stream);
  return launch_forward<double>(*a, (cudaStream_t)stream);
}

extern "C" int64_t jxb_sim_smem_bytes(const JxbSimArgs* a, int backward) {
  if (!a) return -1;
  if (a->dtype == JXB_F32) return (int64_t)sim_smem_layout<float>(*a, backward != 0, nullptr, nullptr);
  return (int64_t)sim_smem_layout<double>(*a, backward != 0, nullptr, nullptr);
}

extern "C" const char* jxb_last_error(void) { return g_err; }
extern "C" int jxb_version(void) { return 1; }
