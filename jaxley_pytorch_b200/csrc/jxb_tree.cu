// Standalone tree solves x = A^{-1} s for a batch of forests (the reference's
// jaxley_pytorch::tree_solve and ::tree_solve_levels ops, kernels/tree_solve.py).
//
//   A[i, i] = d[i],  A[i, p] = l[i],  A[p, i] = u[i]   (p = parent of i)
//
// Arrays are (batch, n) in the caller's node order: every tree a contiguous range,
// root first, parents before children (the DHS solve order).
//
// levels:    one CTA per block of whole trees and batch row. The block's d, s and
//            off-diagonals are staged in shared memory in chain order; one thread
//            eliminates a chain (a node and its only child) bottom-up, chains of a
//            level in parallel, one barrier per chain level; back-substitution
//            top-down. The solution is written back in the caller's order.
// registers: one warp per block of whole trees (at most 32 * R nodes, R <= 8) and
//            batch row; node j lives in lane j % 32, register j / 32. Elimination by
//            node height and back-substitution by depth exchange values with warp
//            shuffles; warps never synchronise with each other. Blocks of 512 to 8192
//            nodes (the reference's largest block, kernels/tree_solve.py:42) use one
//            CTA per block and row instead, exchanging through shared memory.
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

// ---------------------------------------------------------------------------------
// levels
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void tree_levels_kernel(const T* __restrict__ d, const T* __restrict__ l,
                                   const T* __restrict__ u, const T* __restrict__ s,
                                   T* __restrict__ x, JxbTreeSchedule sc) {
  extern __shared__ __align__(16) char smem_raw[];
  const int blk = blockIdx.x;
  const int64_t row = blockIdx.y;
  const int tid = threadIdx.x, NT = blockDim.x;
  const int n0 = sc.block_info[4 * blk + 0];
  const int nn = sc.block_info[4 * blk + 1];
  const int c0 = sc.block_info[4 * blk + 2];
  const int lp0 = sc.block_info[4 * blk + 3];
  const int nlev = sc.block_levels[blk];
  const int cap = sc.max_block_nodes;
  T* D = (T*)smem_raw;
  T* S = D + cap;
  T* AL = S + cap;
  T* AU = AL + cap;
  const int64_t base = row * sc.n_nodes + n0;
  // Stage in chain order: position k holds node perm[n0 + k].
  for (int k = tid; k < nn; k += NT) {
    const int i = sc.perm[n0 + k] - n0;
    D[k] = d[base + i];
    S[k] = s[base + i];
    AL[k] = l[base + i];
    AU[k] = u[base + i];
  }
  __syncthreads();
  const int* lp = sc.level_ptr + lp0;
  for (int h = 0; h < nlev; ++h) {
    for (int c = c0 + lp[h] + tid; c < c0 + lp[h + 1]; c += NT) {
      const int top = sc.chain_top[c];
      const int bot = top + sc.chain_len[c] - 1;
      T dd = D[bot], ss = S[bot];
      for (int k = sc.chain_cptr[c]; k < sc.chain_cptr[c + 1]; ++k) {
        const int ct = sc.chain_child[k];
        const T f = AU[ct] * D[ct];  // D holds reciprocal pivots of eliminated nodes
        dd -= AL[ct] * f;
        ss -= S[ct] * f;
      }
      T id = T(1) / dd;
      D[bot] = id;
      S[bot] = ss;
      for (int j = bot - 1; j >= top; --j) {
        const T f = AU[j + 1] * id;
        dd = D[j] - AL[j + 1] * f;
        ss = S[j] - ss * f;
        id = T(1) / dd;
        D[j] = id;
        S[j] = ss;
      }
    }
    __syncthreads();
  }
  for (int h = nlev - 1; h >= 0; --h) {
    for (int c = c0 + lp[h] + tid; c < c0 + lp[h + 1]; c += NT) {
      const int top = sc.chain_top[c];
      const int bot = top + sc.chain_len[c] - 1;
      const int pt = sc.chain_ptop[c];
      T xp = pt >= 0 ? S[pt] : T(0);
      for (int j = top; j <= bot; ++j) {
        const T v = (S[j] - AL[j] * xp) * D[j];
        S[j] = v;
        xp = v;
      }
    }
    __syncthreads();
  }
  for (int k = tid; k < nn; k += NT) x[base + sc.perm[n0 + k] - n0] = S[k];
}

template <typename T>
int launch_levels(const void* d, const void* l, const void* u, const void* s, void* x,
                  int64_t batch, const JxbTreeSchedule& sc, cudaStream_t st) {
  const size_t smem = 4 * sizeof(T) * (size_t)sc.max_block_nodes;
  if (smem > 227 * 1024) {
    snprintf(g_err, sizeof(g_err), "tree block of %d nodes exceeds shared memory",
             sc.max_block_nodes);
    return JXB_ERR_TOO_LARGE;
  }
  if (batch > 65535) {
    snprintf(g_err, sizeof(g_err), "batch %lld exceeds the grid", (long long)batch);
    return JXB_ERR_ARG;
  }
  cudaError_t e = cudaFuncSetAttribute(tree_levels_kernel<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute", e);
    return JXB_ERR_LAUNCH;
  }
  dim3 grid(sc.n_blocks, (unsigned)batch);
  const int threads = sc.max_block_nodes >= 2048 ? 256 : 128;
  tree_levels_kernel<T><<<grid, threads, smem, st>>>((const T*)d, (const T*)l, (const T*)u,
                                                     (const T*)s, (T*)x, sc);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("tree_levels_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

// ---------------------------------------------------------------------------------
// registers
// ---------------------------------------------------------------------------------
// Value of node `node` (lane node % 32, register node / 32) from every lane.
template <typename T, int R>
__device__ __forceinline__ T gather(const T (&v)[R], int node) {
  const int src = node & 31, reg = node >> 5;
  T out = T(0);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const T w = __shfl_sync(0xffffffffu, v[r], src);
    if (r == reg) out = w;
  }
  return out;
}

template <typename T, int R>
__global__ void tree_registers_kernel(const T* __restrict__ d, const T* __restrict__ l,
                                      const T* __restrict__ u, const T* __restrict__ s,
                                      T* __restrict__ x, JxbRegSchedule sc, int64_t batch) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int nblk = sc.n_blocks;
  if (warp >= nblk * batch) return;  // whole warps exit together
  const int blk = warp % nblk;
  const int64_t row = warp / nblk;
  const int start = sc.block_info[4 * blk + 0];
  const int len = sc.block_info[4 * blk + 1];
  const int levels = sc.block_info[4 * blk + 2];
  const int depth = sc.block_info[4 * blk + 3];
  const int W = 32 * R;
  const int* par = sc.rel_parent + (size_t)blk * W;
  const int* hgt = sc.rel_height + (size_t)blk * W;
  const int* dep = sc.rel_depth + (size_t)blk * W;
  const int* kid = sc.rel_children + (size_t)blk * sc.num_slots * W;
  const int64_t base = row * sc.n_nodes + start;
  T dv[R], sv[R], lv[R], uv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = lane + 32 * r;
    const bool in = j < len;
    dv[r] = in ? d[base + j] : T(1);
    sv[r] = in ? s[base + j] : T(0);
    lv[r] = in ? l[base + j] : T(0);
    uv[r] = in ? u[base + j] : T(0);
  }
  // Elimination by height (leaves have height 0); a node of height h gathers its
  // children's eliminated contributions.
  for (int h = 1; h <= levels; ++h) {
    T al[R], be[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const T f = uv[r] / dv[r];
      al[r] = lv[r] * f;
      be[r] = sv[r] * f;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = lane + 32 * r;
      const bool mine = j < len && hgt[j] == h;
      T ad = T(0), as = T(0);
      for (int k = 0; k < sc.num_slots; ++k) {
        const int c = kid[k * W + j];
        const int cc = c >= 0 ? c : 0;
        const T a1 = gather<T, R>(al, cc);
        const T b1 = gather<T, R>(be, cc);
        if (c >= 0) {
          ad += a1;
          as += b1;
        }
      }
      if (mine) {
        dv[r] -= ad;
        sv[r] -= as;
      }
    }
  }
  // Back-substitution by depth from the roots.
  T xv[R];
#pragma unroll
  for (int r = 0; r < R; ++r) xv[r] = sv[r] / dv[r];
  for (int k = 1; k <= depth; ++k) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = lane + 32 * r;
      const int p = par[j];
      const T xp = gather<T, R>(xv, p);
      if (j < len && dep[j] == k) xv[r] = (sv[r] - lv[r] * xp) / dv[r];
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = lane + 32 * r;
    if (j < len) x[base + j] = xv[r];
  }
}

// Blocks of more than 256 nodes: one CTA of NT threads per block and batch row,
// node j in thread j % NT, register j / NT (R registers a thread for the pivot and
// the right-hand side). A node's eliminated contribution (lower * upper / pivot and
// rhs * upper / pivot) goes to shared memory once, on the level after its own
// elimination, where its parent gathers it; the back-substitution passes the
// parents' solutions through shared memory the same way. One barrier per height
// and per depth level. A thread's off-diagonals and depths are loaded into registers
// with its pivots and right-hand sides before the first level, so that no level
// waits on a global load.
template <typename T, int R, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) tree_registers_cta_kernel(const T* __restrict__ d, const T* __restrict__ l,
                                                                  const T* __restrict__ u, const T* __restrict__ s,
                                                                  T* __restrict__ x, JxbRegSchedule sc) {
  extern __shared__ __align__(16) char smem_raw[];
  const int blk = blockIdx.x;
  const int64_t row = blockIdx.y;
  const int tid = threadIdx.x, NT = blockDim.x;
  const int W = NT * R;
  T* A = (T*)smem_raw;  // W: lower * upper / pivot of eliminated nodes
  T* Bv = A + W;        // W: rhs * upper / pivot, later the solution
  const int start = sc.block_info[4 * blk + 0];
  const int len = sc.block_info[4 * blk + 1];
  const int levels = sc.block_info[4 * blk + 2];
  const int depth = sc.block_info[4 * blk + 3];
  const int* par = sc.rel_parent + (size_t)blk * W;
  const int* hgt = sc.rel_height + (size_t)blk * W;
  const int* dep = sc.rel_depth + (size_t)blk * W;
  const int* kid = sc.rel_children + (size_t)blk * sc.num_slots * W;
  const int64_t base = row * sc.n_nodes + start;
  T dv[R], sv[R], lv[R], uv[R];
  int hv[R], dp[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = tid + NT * r;
    const bool in = j < len;
    dv[r] = in ? d[base + j] : T(1);
    sv[r] = in ? s[base + j] : T(0);
    lv[r] = in ? l[base + j] : T(0);
    uv[r] = in ? u[base + j] : T(0);
    hv[r] = in ? hgt[j] : -1;
    dp[r] = in ? dep[j] : -1;
  }
  for (int h = 1; h <= levels; ++h) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = tid + NT * r;
      if (hv[r] == h - 1) {  // eliminated on the previous level (leaves: height 0)
        const T f = uv[r] / dv[r];
        A[j] = lv[r] * f;
        Bv[j] = sv[r] * f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = tid + NT * r;
      if (hv[r] == h) {
        for (int k = 0; k < sc.num_slots; ++k) {
          const int c = kid[k * W + j];
          if (c >= 0) {
            dv[r] -= A[c];
            sv[r] -= Bv[c];
          }
        }
      }
    }
  }
  __syncthreads();  // every contribution read before Bv holds solutions
  for (int k = 0; k <= depth; ++k) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = tid + NT * r;
      if (dp[r] == k) {
        const T xp = k > 0 ? Bv[par[j]] : T(0);
        sv[r] = (sv[r] - lv[r] * xp) / dv[r];
        Bv[j] = sv[r];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = tid + NT * r;
    if (j < len) x[base + j] = sv[r];
  }
}

template <typename T>
int launch_registers_cta(const void* d, const void* l, const void* u, const void* s, void* x,
                         int64_t batch, const JxbRegSchedule& sc, cudaStream_t st) {
  constexpr int R = 8;
  const int W = 32 * sc.regs_per_lane;  // 512 .. 8192
  const int threads = W / R;
  const size_t smem = 2 * sizeof(T) * (size_t)W;
  if (batch > 65535) {
    snprintf(g_err, sizeof(g_err), "batch %lld exceeds the grid", (long long)batch);
    return JXB_ERR_ARG;
  }
  // up to 512 threads (blocks of up to 4096 nodes) with up to 128 registers, so that a
  // thread's eight nodes stay in registers; 1024 threads at 64
  void (*kern)(const T*, const T*, const T*, const T*, T*, JxbRegSchedule) =
      threads <= 512 ? tree_registers_cta_kernel<T, R, 512> : tree_registers_cta_kernel<T, R, 1024>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    set_err("cudaFuncSetAttribute", e);
    return JXB_ERR_LAUNCH;
  }
  dim3 grid(sc.n_blocks, (unsigned)batch);
  kern<<<grid, threads, smem, st>>>((const T*)d, (const T*)l, (const T*)u, (const T*)s, (T*)x, sc);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("tree_registers_cta_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

template <typename T, int R>
int launch_registers_r(const void* d, const void* l, const void* u, const void* s, void* x,
                       int64_t batch, const JxbRegSchedule& sc, cudaStream_t st) {
  const int64_t warps = (int64_t)sc.n_blocks * batch;
  const int threads = 128;
  const int64_t blocks = (warps * 32 + threads - 1) / threads;
  if (blocks > 0x7fffffff) return JXB_ERR_ARG;
  tree_registers_kernel<T, R><<<(unsigned)blocks, threads, 0, st>>>(
      (const T*)d, (const T*)l, (const T*)u, (const T*)s, (T*)x, sc, batch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err("tree_registers_kernel", e);
    return JXB_ERR_LAUNCH;
  }
  return JXB_OK;
}

template <typename T>
int launch_registers(const void* d, const void* l, const void* u, const void* s, void* x,
                     int64_t batch, const JxbRegSchedule& sc, cudaStream_t st) {
  switch (sc.regs_per_lane) {
    case 1: return launch_registers_r<T, 1>(d, l, u, s, x, batch, sc, st);
    case 2: return launch_registers_r<T, 2>(d, l, u, s, x, batch, sc, st);
    case 4: return launch_registers_r<T, 4>(d, l, u, s, x, batch, sc, st);
    case 8: return launch_registers_r<T, 8>(d, l, u, s, x, batch, sc, st);
    case 16:
    case 32:
    case 64:
    case 128:
    case 256: return launch_registers_cta<T>(d, l, u, s, x, batch, sc, st);
    default:
      snprintf(g_err, sizeof(g_err), "regs_per_lane must be a power of two from 1 to 256");
      return JXB_ERR_ARG;
  }
}

}  // namespace

extern "C" int jxb_tree_solve_levels(int dtype, const void* d, const void* l, const void* u,
                                     const void* s, void* x, int64_t batch,
                                     const JxbTreeSchedule* sc, void* stream) {
  if (!sc || !d || !l || !u || !s || !x || batch < 0) return JXB_ERR_ARG;
  if (batch == 0 || sc->n_blocks == 0) return JXB_OK;
  if (dtype == JXB_F32) return launch_levels<float>(d, l, u, s, x, batch, *sc, (cudaStream_t)stream);
  if (dtype == JXB_F64) return launch_levels<double>(d, l, u, s, x, batch, *sc, (cudaStream_t)stream);
  return JXB_ERR_DTYPE;
}

extern "C" int jxb_tree_solve_registers(int dtype, const void* d, const void* l, const void* u,
                                        const void* s, void* x, int64_t batch,
                                        const JxbRegSchedule* sc, void* stream) {
  if (!sc || !d || !l || !u || !s || !x || batch < 0) return JXB_ERR_ARG;
  if (batch == 0 || sc->n_blocks == 0) return JXB_OK;
  if (dtype == JXB_F32) return launch_registers<float>(d, l, u, s, x, batch, *sc, (cudaStream_t)stream);
  if (dtype == JXB_F64) return launch_registers<double>(d, l, u, s, x, batch, *sc, (cudaStream_t)stream);
  return JXB_ERR_DTYPE;
}
