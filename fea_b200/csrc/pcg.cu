// Jacobi-preconditioned CG on the reduced CSR stiffness (sm_100a).
//
// Replaces the reference's linear solve (FEA = sssnnn7119/FEA):
//   StaticImplicitSolver._solve_linear_equation  static_implicit.py:352-405
//     d = sqrt|diag K|, K~ = D^-1 K D^-1, b~ = D^-1 b, x0~ = D x0
//   _linear_solver.conjugate_gradient            _linear_solver.py:6-42
//     plain CG on K~ with stop test ||r~||^2 / ||b~||^2 < tol
// CG on the symmetrically scaled system is Jacobi-PCG on K with
// M = |diag K| (x = D^-1 x~, r = D r~), so this file runs PCG directly and
// evaluates the same stop test as (r.M^-1 r) / (b.M^-1 b).
//
// One iteration = 3 kernels: (1) q = K p fused with p.q, (2) x, r, z update
// fused with r.z, (3) p update.  Scalars (alpha, beta, r.z, status) stay on
// the device; every dot product is a fixed-order two-level sum (per-block
// partials over a fixed grid, summed by the last block to finish), so
// results are bitwise reproducible.  The host reads the status every
// `check_every` iterations.
//
// Two SpMV operators:
//   CsrOp  — any CSR matrix; LANES threads per row.
//   NodeOp — the plan's reduced matrix: the f free rows of node n are
//            consecutive, share one column list of length L_n and sit at
//            vbase[n] + j * L_n in the values.  One warp per node reads the
//            column indices and gathers x once for all f rows, so index
//            traffic is nnz / f * 4 bytes instead of nnz * 4.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>
#include <unordered_map>

#include "common.cuh"

namespace fea {

constexpr int PCG_TPB = 256;
constexpr int PCG_WARPS = PCG_TPB / 32;
constexpr int PCG_GRID = 148 * 8;   // fixed grid: bounds the partial count

// device-side solver state (doubles, in the work buffer)
enum { S_RZ = 0, S_RZ0, S_ALPHA, S_BETA, S_DONE, S_ITER, S_STATUS, S_PQ, S_COUNT, S_LEN = 16 };

template <class V>
struct CsrOp {
  const int64_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const V* __restrict__ val;
  int64_t n;      // rows
  int64_t nnz;
};

template <class V>
struct NodeOp {
  const int64_t* __restrict__ vbase;
  const int32_t* __restrict__ rowlen;
  const int32_t* __restrict__ dbase;
  const uint8_t* __restrict__ mask;
  const int32_t* __restrict__ idx;
  const V* __restrict__ val;
  int64_t n_nodes;
  int64_t n;      // rows (free DOFs)
};

// block sum: warp shuffles, then the 8 warp sums in fixed order
__device__ __forceinline__ double block_sum_w(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < PCG_WARPS; ++i) r += sh[i];
  __syncthreads();
  return r;
}

// last-block-done reduction of per-block partials in block order
__device__ __forceinline__ bool last_block(unsigned* counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned prev = atomicAdd(counter, 1u);
    last = prev == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}

// sum of n (<= a few thousand) partials written by other blocks of this
// grid; L2 loads (.cg) issued back to back, fixed order per thread
__device__ __forceinline__ double sum_partials(const double* part, int n, int stride, int off, double* sh) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int i = threadIdx.x;
  for (; i + 3 * PCG_TPB < n; i += 4 * PCG_TPB) {
    a0 += __ldcg(part + (int64_t)i * stride + off);
    a1 += __ldcg(part + (int64_t)(i + PCG_TPB) * stride + off);
    a2 += __ldcg(part + (int64_t)(i + 2 * PCG_TPB) * stride + off);
    a3 += __ldcg(part + (int64_t)(i + 3 * PCG_TPB) * stride + off);
  }
  for (; i < n; i += PCG_TPB) a0 += __ldcg(part + (int64_t)i * stride + off);
  return block_sum_w((a0 + a1) + (a2 + a3), sh);
}

// PCG step 1 epilogue: alpha = rz / p.q (or breakdown)
__device__ __forceinline__ void finish_pq(double contrib, double* st, double* part, unsigned* counter) {
  __shared__ double sh[PCG_WARPS];
  double bs = block_sum_w(contrib, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
  if (last_block(counter)) {
    double pq = sum_partials(part, gridDim.x, 1, 0, sh);
    if (threadIdx.x == 0) {
      st[S_PQ] = pq;
      if (!(pq > 0.0) || !isfinite(pq)) {
        st[S_STATUS] = (double)FEA_EBREAKDOWN;
        st[S_DONE] = 1.0;
        st[S_ALPHA] = 0.0;
      } else {
        st[S_ALPHA] = st[S_RZ] / pq;
      }
      *counter = 0u;
    }
  }
}

// ---- CSR operator: LANES threads per row, warp-uniform loop ----------------
// y = A x ; mode 1: also p.q partials and the alpha epilogue
template <int LANES, class V, class X>
__global__ void __launch_bounds__(PCG_TPB) k_spmv_csr(CsrOp<V> A, const X* __restrict__ x, X* __restrict__ y,
                                                      double* st, double* part, unsigned* counter, int mode) {
  if (mode == 1 && st[S_DONE] != 0.0) return;
  constexpr int RPW = 32 / LANES;                 // rows per warp
  const int lane = threadIdx.x % LANES;
  const int warp = threadIdx.x >> 5;
  const int sub = (threadIdx.x & 31) / LANES;
  double contrib = 0.0;
  for (int64_t base = ((int64_t)blockIdx.x * PCG_WARPS + warp) * RPW; base < A.n;
       base += (int64_t)gridDim.x * PCG_WARPS * RPW) {
    const int64_t row = base + sub;
    double s = 0.0;
    if (row < A.n) {
      const int64_t b = A.ptr[row], e = A.ptr[row + 1];
      for (int64_t i = b + lane; i < e; i += LANES) s += (double)A.val[i] * (double)x[A.idx[i]];
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
    if (row < A.n && lane == 0) {
      y[row] = (X)s;
      contrib += s * (double)x[row];
    }
  }
  if (mode == 1) finish_pq(contrib, st, part, counter);
}

// ---- node operator: one warp per node row block ------------------------------
template <class V, class X>
__global__ void __launch_bounds__(PCG_TPB) k_spmv_node(NodeOp<V> A, const X* __restrict__ x, X* __restrict__ y,
                                                       double* st, double* part, unsigned* counter, int mode) {
  if (mode == 1 && st[S_DONE] != 0.0) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t step = (int64_t)gridDim.x * PCG_WARPS;
  double contrib = 0.0;
  // One warp walks nodes nd, nd + step, ...  The metadata and the first 96
  // column indices of the next node are loaded while the current node is
  // processed, so its gathers of x need not wait for a DRAM round trip.
  int64_t nd = (int64_t)blockIdx.x * PCG_WARPS + warp;
  unsigned m = 0;
  int L = 0;
  int64_t vb = 0;
  int32_t jn[3] = {0, 0, 0};
  if (nd < A.n_nodes) {
    m = A.mask[nd];
    L = m ? A.rowlen[nd] : 0;
    vb = A.vbase[nd];
#pragma unroll
    for (int k = 0; k < 3; ++k) jn[k] = lane + 32 * k < L ? __ldg(A.idx + vb + lane + 32 * k) : 0;
  }
  while (nd < A.n_nodes) {
    const int64_t nx = nd + step;
    unsigned m2 = 0;
    int L2 = 0;
    int64_t vb2 = 0;
    if (nx < A.n_nodes) {
      m2 = A.mask[nx];
      L2 = A.rowlen[nx];
      vb2 = A.vbase[nx];
    }
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const int f = popc3(m);
    if (m) {                                        // warp-uniform
      const V* __restrict__ v0 = A.val + vb;
      // 96 columns per pass: values issued first, then the gathers of x
      // (L2-resident), then the FMAs
      for (int q0 = 0; q0 < L; q0 += 96) {
        int32_t j[3];
        bool h[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int q = q0 + lane + 32 * k;
          h[k] = q < L;
          j[k] = q0 == 0 ? jn[k] : (h[k] ? __ldg(A.idx + vb + q) : 0);
        }
        double va[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int q = q0 + lane + 32 * k;
            va[r][k] = (r < f && h[k]) ? (double)__ldcs(v0 + (int64_t)r * L + q) : 0.0;
          }
        double xv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) xv[k] = h[k] ? (double)x[j[k]] : 0.0;
        s0 += va[0][0] * xv[0] + va[0][1] * xv[1] + va[0][2] * xv[2];
        s1 += va[1][0] * xv[0] + va[1][1] * xv[1] + va[1][2] * xv[2];
        s2 += va[2][0] * xv[0] + va[2][1] * xv[1] + va[2][2] * xv[2];
      }
    }
    // column indices of the next node's first pass
    const int Ln = m2 ? L2 : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) jn[k] = lane + 32 * k < Ln ? __ldg(A.idx + vb2 + lane + 32 * k) : 0;
    if (m) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      }
      if (lane == 0) {
        const int64_t r = A.dbase[nd];
        y[r] = (X)s0;
        contrib += s0 * (double)x[r];
        if (f > 1) { y[r + 1] = (X)s1; contrib += s1 * (double)x[r + 1]; }
        if (f > 2) { y[r + 2] = (X)s2; contrib += s2 * (double)x[r + 2]; }
      }
    }
    nd = nx;
    m = m2;
    L = Ln;
    vb = vb2;
  }
  if (mode == 1) finish_pq(contrib, st, part, counter);
}

// Node rows with LPN < 32 lanes per node (32 / LPN nodes per warp), CPL
// columns per lane per pass: more nodes, and more loads, in flight per warp;
// used for the FP32 values of the mixed solver, whose 4-byte loads leave the
// one-node-per-warp kernel latency-bound.  The next nodes' metadata and
// first-pass column indices are loaded while the current nodes are
// processed.  Used with LPN = 16, CPL = 3 (48-column passes): 96-column
// passes (CPL = 6) need 77 registers, 3 CTAs per SM, and ran the FP32
// iteration 0.237 ms against 0.134 ms at 64^3.  Loops and shuffles
// warp-uniform.
template <int LPN, int CPL, class V, class X>
__global__ void __launch_bounds__(PCG_TPB) k_spmv_node_sub(NodeOp<V> A, const X* __restrict__ x, X* __restrict__ y,
                                                           double* st, double* part, unsigned* counter, int mode) {
  if (mode == 1 && st[S_DONE] != 0.0) return;
  constexpr int NPW = 32 / LPN;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane / LPN, hl = lane % LPN;
  const int64_t step = (int64_t)gridDim.x * PCG_WARPS * NPW;
  double contrib = 0.0;
  int64_t base = ((int64_t)blockIdx.x * PCG_WARPS + warp) * NPW;
  int64_t nd = base + sub;
  unsigned m = 0;
  int L = 0;
  int64_t vb = 0;
  int32_t db = 0;
  int32_t jn[CPL];
#pragma unroll
  for (int k = 0; k < CPL; ++k) jn[k] = 0;
  if (nd < A.n_nodes) {
    m = A.mask[nd];
    L = m ? A.rowlen[nd] : 0;
    vb = A.vbase[nd];
    db = A.dbase[nd];
#pragma unroll
    for (int k = 0; k < CPL; ++k) jn[k] = hl + LPN * k < L ? __ldg(A.idx + vb + hl + LPN * k) : 0;
  }
  for (; base < A.n_nodes; base += step) {                  // warp-uniform
    const int64_t nx = nd + step;
    unsigned m2 = 0;
    int L2 = 0;
    int64_t vb2 = 0;
    int32_t db2 = 0;
    if (nx < A.n_nodes) {
      m2 = A.mask[nx];
      L2 = A.rowlen[nx];
      vb2 = A.vbase[nx];
      db2 = A.dbase[nx];
    }
    const int f = popc3(m);
    int Lmax = L;
#pragma unroll
    for (int o = 16; o >= LPN; o >>= 1) Lmax = max(Lmax, __shfl_xor_sync(0xffffffffu, Lmax, o));
    const V* __restrict__ v0 = A.val + vb;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int q0 = 0; q0 < Lmax; q0 += CPL * LPN) {
      int32_t j[CPL];
      bool h[CPL];
#pragma unroll
      for (int k = 0; k < CPL; ++k) {
        const int q = q0 + hl + LPN * k;
        h[k] = q < L;
        j[k] = q0 == 0 ? jn[k] : (h[k] ? __ldg(A.idx + vb + q) : 0);
      }
      double va[3][CPL];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
          const int q = q0 + hl + LPN * k;
          va[r][k] = (r < f && h[k]) ? (double)__ldcs(v0 + (int64_t)r * L + q) : 0.0;
        }
      double xv[CPL];
#pragma unroll
      for (int k = 0; k < CPL; ++k) xv[k] = h[k] ? (double)x[j[k]] : 0.0;
      if constexpr (CPL == 3) {
        s0 += va[0][0] * xv[0] + va[0][1] * xv[1] + va[0][2] * xv[2];
        s1 += va[1][0] * xv[0] + va[1][1] * xv[1] + va[1][2] * xv[2];
        s2 += va[2][0] * xv[0] + va[2][1] * xv[1] + va[2][2] * xv[2];
      } else {
#pragma unroll
        for (int k = 0; k < CPL; ++k) {
          s0 += va[0][k] * xv[k];
          s1 += va[1][k] * xv[k];
          s2 += va[2][k] * xv[k];
        }
      }
    }
    const int Ln = m2 ? L2 : 0;
#pragma unroll
    for (int k = 0; k < CPL; ++k) jn[k] = hl + LPN * k < Ln ? __ldg(A.idx + vb2 + hl + LPN * k) : 0;
#pragma unroll
    for (int o = LPN / 2; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o, LPN);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o, LPN);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o, LPN);
    }
    if (m && hl < f) {
      const int64_t r = db + hl;
      const double sr = hl == 0 ? s0 : (hl == 1 ? s1 : s2);
      y[r] = (X)sr;
      contrib += sr * (double)x[r];
    }
    nd = nx;
    m = m2;
    L = Ln;
    vb = vb2;
    db = db2;
  }
  if (mode == 1) finish_pq(contrib, st, part, counter);
}

// FP32 copy of the node-row matrix in a padded layout: every node's column
// list and each of its rows start on a 16-byte boundary and are padded to a
// multiple of 4 entries (column 0, value 0), so that a lane reads 4 columns
// and the 4 values of each row with 128-bit loads.
struct NodeOp32q {
  const int64_t* __restrict__ cbase;   // [N+1] first padded column of node n
  const int64_t* __restrict__ qbase;   // [N+1] first value of node n's rows
  const int32_t* __restrict__ cols;
  const float* __restrict__ vals;
  const uint8_t* __restrict__ mask;
  const int32_t* __restrict__ dbase;
  int64_t n_nodes;
  int64_t n;
};

// LPN lanes per node (32 / LPN nodes per warp), 4 columns per lane per
// pass: the next nodes' metadata are loaded while the current ones are
// processed; loops and shuffles warp-uniform.
#ifndef FEA_F32Q_LPN
#define FEA_F32Q_LPN 8
#endif
template <int LPN, class X>
__global__ void __launch_bounds__(PCG_TPB, 4) k_spmv_node32q(NodeOp32q A, const X* __restrict__ x, X* __restrict__ y,
                                                             double* st, double* part, unsigned* counter, int mode) {
  if (mode == 1 && st[S_DONE] != 0.0) return;
  constexpr int NPW = 32 / LPN;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane / LPN, hl = lane % LPN;
  const int64_t step = (int64_t)gridDim.x * PCG_WARPS * NPW;
  double contrib = 0.0;
  int64_t base = ((int64_t)blockIdx.x * PCG_WARPS + warp) * NPW;
  int64_t nd = base + sub;
  unsigned m = 0;
  int64_t cb = 0, ce = 0, qb = 0;
  int32_t db = 0;
  if (nd < A.n_nodes) {
    m = A.mask[nd];
    cb = A.cbase[nd];
    ce = A.cbase[nd + 1];
    qb = A.qbase[nd];
    db = A.dbase[nd];
  }
  for (; base < A.n_nodes; base += step) {       // warp-uniform
    const int64_t nx = nd + step;
    unsigned m2 = 0;
    int64_t cb2 = 0, ce2 = 0, qb2 = 0;
    int32_t db2 = 0;
    if (nx < A.n_nodes) {                        // the next nodes' metadata, loaded ahead
      m2 = A.mask[nx];
      cb2 = A.cbase[nx];
      ce2 = A.cbase[nx + 1];
      qb2 = A.qbase[nx];
      db2 = A.dbase[nx];
    }
    const int f = popc3(m);
    const int L4 = m ? (int)(ce - cb) : 0;
    int Lmax = L4;
#pragma unroll
    for (int o = 16; o >= LPN; o >>= 1) Lmax = max(Lmax, __shfl_xor_sync(0xffffffffu, Lmax, o));
    // FP32 products and row sums (the inner solve is FP32; its residual is
    // refined in FP64), FP64 for the p.q contribution
    float s0 = 0.f, s1 = 0.f, s2 = 0.f;
    for (int q0 = 0; q0 < Lmax; q0 += 4 * LPN) {
      const int q = q0 + 4 * hl;
      const bool h = q < L4;
      const int4 c = h ? __ldg(reinterpret_cast<const int4*>(A.cols + cb + q)) : make_int4(0, 0, 0, 0);
      const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 v0 = h ? __ldcs(reinterpret_cast<const float4*>(A.vals + qb + q)) : z4;
      const float4 v1 = (h && f > 1) ? __ldcs(reinterpret_cast<const float4*>(A.vals + qb + L4 + q)) : z4;
      const float4 v2 = (h && f > 2) ? __ldcs(reinterpret_cast<const float4*>(A.vals + qb + 2 * L4 + q)) : z4;
      float x0 = 0.f, x1 = 0.f, x2 = 0.f, x3 = 0.f;
      if (h) {
        x0 = (float)x[c.x];
        x1 = (float)x[c.y];
        x2 = (float)x[c.z];
        x3 = (float)x[c.w];
      }
      s0 += v0.x * x0 + v0.y * x1 + v0.z * x2 + v0.w * x3;
      s1 += v1.x * x0 + v1.y * x1 + v1.z * x2 + v1.w * x3;
      s2 += v2.x * x0 + v2.y * x1 + v2.z * x2 + v2.w * x3;
    }
#pragma unroll
    for (int o = LPN / 2; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o, LPN);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o, LPN);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o, LPN);
    }
    if (m && hl < f) {
      const int64_t r = db + hl;
      const double sr = (double)(hl == 0 ? s0 : (hl == 1 ? s1 : s2));
      y[r] = (X)sr;
      contrib += sr * (double)x[r];
    }
    nd = nx;
    m = m2;
    cb = cb2;
    ce = ce2;
    qb = qb2;
    db = db2;
  }
  if (mode == 1) finish_pq(contrib, st, part, counter);
}

// Fill the padded FP32 layout from the FP64 node-row values (and, when
// cols != nullptr, the padded column lists): one warp per node.
__global__ void __launch_bounds__(256) k_fill_node32q(NodeOp<double> A, const int64_t* __restrict__ cbase,
                                                      const int64_t* __restrict__ qbase, int32_t* cols,
                                                      float* __restrict__ vals) {
  const int lane = threadIdx.x & 31;
  const int64_t nd = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (nd >= A.n_nodes) return;
  const unsigned m = A.mask[nd];
  if (!m) return;
  const int f = popc3(m);
  const int L = A.rowlen[nd];
  const int64_t vb = A.vbase[nd], cb = cbase[nd], qb = qbase[nd];
  const int L4 = (int)(cbase[nd + 1] - cb);
  for (int q = lane; q < L4; q += 32) {
    if (cols) cols[cb + q] = q < L ? A.idx[vb + q] : 0;
    for (int r = 0; r < f; ++r) vals[qb + (int64_t)r * L4 + q] = q < L ? (float)A.val[vb + (int64_t)r * L + q] : 0.f;
  }
}

// 1/|K_jj| of the node rows (0 -> 1): the diagonal entry of row (n, j) is the
// column dbase[n] + j of the shared column list (sorted), found by bisection
template <class V>
__global__ void k_dinv_node(NodeOp<V> A, double* __restrict__ dinv) {
  const int64_t nd = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (nd >= A.n_nodes) return;
  const unsigned m = A.mask[nd];
  const int f = popc3(m);
  const int L = A.rowlen[nd];
  const int64_t vb = A.vbase[nd];
  const int32_t r0 = A.dbase[nd];
  for (int j = 0; j < f; ++j) {
    int lo = 0, hi = L;
    double dv = 0.0;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const int32_t c = A.idx[vb + mid];
      if (c == r0 + j) { dv = (double)A.val[vb + (int64_t)j * L + mid]; break; }
      if (c < r0 + j) lo = mid + 1; else hi = mid;
    }
    dv = fabs(dv);
    dinv[r0 + j] = dv == 0.0 ? 1.0 : 1.0 / dv;
  }
}

template <class V>
__global__ void k_dinv_csr(CsrOp<V> A, double* __restrict__ dinv, int identity) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += (int64_t)gridDim.x * blockDim.x) {
    if (identity) { dinv[i] = 1.0; continue; }
    int64_t lo = A.ptr[i], hi = A.ptr[i + 1];
    double dv = 0.0;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int32_t c = A.idx[mid];
      if (c == i) { dv = (double)A.val[mid]; break; }
      if (c < i) lo = mid + 1; else hi = mid;
    }
    dv = fabs(dv);
    dinv[i] = dv == 0.0 ? 1.0 : 1.0 / dv;
  }
}

// x += alpha p; r -= alpha q; z = r / |d|; partial r.z; last block: beta, stop test.
// Each thread takes PCG_VU rows a grid stride apart and issues all their
// loads before any arithmetic (one resident wave covers the vector in one
// pass up to PCG_VU x 303k rows), so the loads of a thread overlap instead
// of paying one round trip per row.
constexpr int PCG_VU = 4;

template <class X>
__global__ void __launch_bounds__(PCG_TPB) k_pcg_update(int64_t n, X* __restrict__ x, X* __restrict__ r,
                                                        X* __restrict__ z, const X* __restrict__ p,
                                                        const X* __restrict__ q, const double* __restrict__ dinv,
                                                        double* st, double* part, unsigned* counter, double tol,
                                                        int max_iter) {
  __shared__ double sh[PCG_WARPS];
  if (st[S_DONE] != 0.0) return;
  const double alpha = st[S_ALPHA];
  double contrib = 0.0;
  const int64_t stride = (int64_t)gridDim.x * PCG_TPB;
  for (int64_t i0 = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i0 < n; i0 += PCG_VU * stride) {
    X xv[PCG_VU], rv[PCG_VU], pv[PCG_VU], qv[PCG_VU];
    double dv[PCG_VU];
#pragma unroll
    for (int u = 0; u < PCG_VU; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < n) {
        xv[u] = x[i];
        rv[u] = r[i];
        pv[u] = p[i];
        qv[u] = q[i];
        dv[u] = dinv[i];
      }
    }
#pragma unroll
    for (int u = 0; u < PCG_VU; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < n) {
        x[i] = (X)((double)xv[u] + alpha * (double)pv[u]);
        const double ri = (double)rv[u] - alpha * (double)qv[u];
        r[i] = (X)ri;
        const double zi = ri * dv[u];
        z[i] = (X)zi;
        contrib += ri * zi;
      }
    }
  }
  double bs = block_sum_w(contrib, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
  if (last_block(counter)) {
    double rz = sum_partials(part, gridDim.x, 1, 0, sh);
    if (threadIdx.x == 0) {
      double it = st[S_ITER] + 1.0;
      st[S_ITER] = it;
      st[S_BETA] = rz / st[S_RZ];
      st[S_RZ] = rz;
      if (!isfinite(rz)) {
        st[S_STATUS] = (double)FEA_EBREAKDOWN;
        st[S_DONE] = 1.0;
      } else if (rz / st[S_RZ0] < tol) {
        st[S_DONE] = 1.0;
      } else if (it >= (double)max_iter) {
        st[S_STATUS] = (double)FEA_ENOTCONV;
        st[S_DONE] = 1.0;
      }
      *counter = 0u;
    }
  }
}

template <class X>
__global__ void __launch_bounds__(PCG_TPB) k_pcg_p(int64_t n, X* __restrict__ p, const X* __restrict__ z,
                                                   const double* st) {
  if (st[S_DONE] != 0.0) return;
  const double beta = st[S_BETA];
  const int64_t stride = (int64_t)gridDim.x * PCG_TPB;
  for (int64_t i0 = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i0 < n; i0 += PCG_VU * stride) {
    X zv[PCG_VU], pv[PCG_VU];
#pragma unroll
    for (int u = 0; u < PCG_VU; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < n) {
        zv[u] = z[i];
        pv[u] = p[i];
      }
    }
#pragma unroll
    for (int u = 0; u < PCG_VU; ++u) {
      const int64_t i = i0 + u * stride;
      if (i < n) p[i] = (X)((double)zv[u] + beta * (double)pv[u]);
    }
  }
}

// setup (dinv given): r = b - Ax (Ax in r on entry), z = dinv r, p = z,
// partial r.z and b.dinv.b; last block initialises the state.
template <class X>
__global__ void __launch_bounds__(PCG_TPB) k_pcg_setup(int64_t n, const double* __restrict__ b, X* __restrict__ r,
                                                       X* __restrict__ z, X* __restrict__ p,
                                                       const double* __restrict__ dinv, double* st, double* part,
                                                       unsigned* counter) {
  __shared__ double sh[PCG_WARPS];
  double c_rz = 0.0, c_bb = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * PCG_TPB) {
    const double di = dinv[i];
    double ri = b[i] - (double)r[i];
    r[i] = (X)ri;
    double zi = ri * di;
    z[i] = (X)zi;
    p[i] = (X)zi;
    c_rz += ri * zi;
    c_bb += b[i] * b[i] * di;
  }
  double s1 = block_sum_w(c_rz, sh);
  double s2 = block_sum_w(c_bb, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
  if (last_block(counter)) {
    double rz = sum_partials(part, gridDim.x, 2, 0, sh);
    double bb = sum_partials(part, gridDim.x, 2, 1, sh);
    if (threadIdx.x == 0) {
      st[S_RZ] = rz;
      st[S_RZ0] = bb;
      st[S_ITER] = 0.0;
      st[S_STATUS] = 0.0;
      // a zero right-hand side or an exact initial guess needs no iteration
      st[S_DONE] = (bb == 0.0 || rz == 0.0) ? 1.0 : 0.0;
      if (bb == 0.0) st[S_RZ0] = 1.0;
      *counter = 0u;
    }
  }
}

__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

__global__ void k_axpy_f32(int64_t n, double* __restrict__ x, const float* __restrict__ d) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)d[i];
}

// Residual replacement of the mixed solver (after x64 += x32, x32 = 0):
// r64 = b - A x64 (A x64 in r64 on entry), r32 = float(r64), z32 =
// float(r32 dinv), and in the last block: the true stop test
// (r64.D^-1 r64)/(b.D^-1 b) into st64, rho' = r32.z32 and beta' = rho' beta /
// rho (the FP32 recurrence continues with the true residual and the same
// search direction), and the FP32 done flag cleared unless the true residual
// has converged.
__global__ void __launch_bounds__(PCG_TPB) k_mixed_replace(int64_t n, const double* __restrict__ b,
                                                           double* __restrict__ r64, const double* __restrict__ dinv,
                                                           float* __restrict__ r32, float* __restrict__ z32,
                                                           double* st64, double* st32, double* part,
                                                           unsigned* counter, double tol) {
  __shared__ double sh[PCG_WARPS];
  double c_rr = 0.0, c_rz = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * PCG_TPB) {
    const double ri = b[i] - r64[i];
    r64[i] = ri;
    const float rf = (float)ri;
    r32[i] = rf;
    const double zi = (double)rf * dinv[i];
    const float zf = (float)zi;
    z32[i] = zf;
    c_rr += ri * ri * dinv[i];
    c_rz += (double)rf * zi;
  }
  const double s1 = block_sum_w(c_rr, sh);
  const double s2 = block_sum_w(c_rz, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
  if (last_block(counter)) {
    const double rr = sum_partials(part, gridDim.x, 2, 0, sh);
    const double rho = sum_partials(part, gridDim.x, 2, 1, sh);
    if (threadIdx.x == 0) {
      st64[S_RZ] = rr;
      const bool conv = rr / st64[S_RZ0] < tol;
      st64[S_DONE] = conv ? 1.0 : 0.0;
      const double rho_old = st32[S_RZ], beta = st32[S_BETA];
      st32[S_BETA] = rho_old != 0.0 ? rho * beta / rho_old : 0.0;
      st32[S_RZ] = rho;
      if (st32[S_STATUS] == 0.0) st32[S_DONE] = conv ? 1.0 : 0.0;
      *counter = 0u;
    }
  }
}

static int lanes_for(int64_t n, int64_t nnz) {
  double avg = n ? (double)nnz / (double)n : 0.0;
  return avg >= 40.0 ? 32 : (avg >= 12.0 ? 16 : 8);
}

// Grid of a PCG kernel: one wave of resident blocks (occupancy x SMs,
// capped at PCG_GRID so the partials fit the work buffer), fewer if there
// are fewer units.  A fixed function of kernel and device, so the partial
// sums keep one order from call to call.
static std::mutex g_occ_mu;
static std::unordered_map<const void*, int> g_occ[64];

template <class Kern>
static unsigned occ_grid(Kern kern, int64_t units, int per_block, int threads = PCG_TPB) {
  int dev = 0;
  cudaGetDevice(&dev);
  int wave = PCG_GRID;
  {
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto& m = g_occ[dev & 63];
    auto it = m.find((const void*)kern);
    if (it != m.end()) {
      wave = it->second;
    } else {
      int sms = 148, nb = 1;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, 0);
      wave = (int)std::min<int64_t>((int64_t)sms * std::max(nb, 1), PCG_GRID);
      m[(const void*)kern] = wave;
    }
  }
  const int64_t need = (units + per_block - 1) / per_block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(need, wave));
}

static unsigned fixed_grid(int64_t units, int per_block) {
  int64_t g = (units + per_block - 1) / per_block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, PCG_GRID));
}

template <class V, class X>
static void spmv(const CsrOp<V>& A, const X* x, X* y, double* st, double* part, unsigned* counter, int mode,
                 cudaStream_t s) {
  const int L = lanes_for(A.n, A.nnz);
  const int rpb = PCG_TPB / L;
  if (L == 32) k_spmv_csr<32, V, X><<<occ_grid(k_spmv_csr<32, V, X>, A.n, rpb), PCG_TPB, 0, s>>>(A, x, y, st, part,
                                                                                            counter, mode);
  else if (L == 16) k_spmv_csr<16, V, X><<<occ_grid(k_spmv_csr<16, V, X>, A.n, rpb), PCG_TPB, 0, s>>>(A, x, y, st,
                                                                                                 part, counter, mode);
  else k_spmv_csr<8, V, X><<<occ_grid(k_spmv_csr<8, V, X>, A.n, rpb), PCG_TPB, 0, s>>>(A, x, y, st, part, counter,
                                                                                  mode);
  count_launch();
}

template <class V, class X>
static void spmv(const NodeOp<V>& A, const X* x, X* y, double* st, double* part, unsigned* counter, int mode,
                 cudaStream_t s) {
  if (sizeof(V) == 4) {
    k_spmv_node_sub<16, 3, V, X><<<occ_grid(k_spmv_node_sub<16, 3, V, X>, A.n_nodes, 2 * PCG_WARPS), PCG_TPB, 0, s>>>(
        A, x, y, st, part, counter, mode);
  } else {
    k_spmv_node<V, X><<<occ_grid(k_spmv_node<V, X>, A.n_nodes, PCG_WARPS), PCG_TPB, 0, s>>>(A, x, y, st, part,
                                                                                          counter, mode);
  }
  count_launch();
}

template <class X>
static void spmv(const NodeOp32q& A, const X* x, X* y, double* st, double* part, unsigned* counter, int mode,
                 cudaStream_t s) {
  constexpr int LPN = FEA_F32Q_LPN;
  k_spmv_node32q<LPN, X><<<occ_grid(k_spmv_node32q<LPN, X>, A.n_nodes, PCG_WARPS * (32 / LPN)), PCG_TPB, 0, s>>>(
      A, x, y, st, part, counter, mode);
  count_launch();
}

template <class V>
static void diag_inv(const CsrOp<V>& A, double* dinv, int jacobi, cudaStream_t s) {
  k_dinv_csr<V><<<fixed_grid(A.n, 256), 256, 0, s>>>(A, dinv, jacobi ? 0 : 1);
  count_launch();
}

template <class V>
static void diag_inv(const NodeOp<V>& A, double* dinv, int, cudaStream_t s) {
  k_dinv_node<V><<<grid_for(A.n_nodes, 128), 128, 0, s>>>(A, dinv);
  count_launch();
}

template <class X>
static unsigned vec_grid(int64_t n) {
  // the update kernel's wave sizes all three vector kernels (same partials)
  return occ_grid(k_pcg_update<X>, n, PCG_TPB);
}

static int64_t part_len(int64_t) { return 2 * PCG_GRID + 2; }

// Work layout (doubles): st[S_LEN] | counter(2) | dinv[n] | r | z | p | q | part
struct PcgWork {
  double* st;
  unsigned* counter;
  double* dinv;
  double *r, *z, *p, *q;
  double* part;
};

static PcgWork carve(double* w, int64_t n) {
  PcgWork W;
  W.st = w;
  W.counter = (unsigned*)(w + S_LEN);
  W.dinv = w + S_LEN + 2;
  W.r = W.dinv + n;
  W.z = W.r + n;
  W.p = W.z + n;
  W.q = W.p + n;
  W.part = W.q + n;
  return W;
}

// Run PCG iterations on (A, b) in precision X starting from x (in X), with
// dinv given.  Returns status; *iters.  A64 computes the FP64 residual of
// the initial guess (same operator in FP64 values).
template <class Op, class X>
static int pcg_core(const Op& A, int64_t n, const double* b, X* x, X* r, X* z, X* p, X* q, const double* dinv,
                    double* st, unsigned* counter, double* part, double tol, int max_iter, int check_every,
                    int* iters, double* relres, cudaStream_t s) {
  spmv(A, (const X*)x, r, st, part, counter, 0, s);       // r = A x
  const unsigned vg = vec_grid<X>(n);
  k_pcg_setup<X><<<vg, PCG_TPB, 0, s>>>(n, b, r, z, p, dinv, st, part, counter);
  count_launch();
  if (cudaError_t e = cudaGetLastError()) return (int)e;
  double host[S_LEN];
  int it_done = 0;
  const int ce = std::max(1, check_every);
  while (true) {
    cudaMemcpyAsync(host, st, sizeof(host), cudaMemcpyDeviceToHost, s);
    if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
    if (host[S_DONE] != 0.0 || it_done >= max_iter) break;
    const int batch = std::min(ce, max_iter - it_done);
    for (int k = 0; k < batch; ++k) {
      spmv(A, (const X*)p, q, st, part, counter, 1, s);
      k_pcg_update<X><<<vg, PCG_TPB, 0, s>>>(n, x, r, z, p, q, dinv, st, part, counter, tol, max_iter);
      k_pcg_p<X><<<vg, PCG_TPB, 0, s>>>(n, p, z, st);
      count_launch(2);
    }
    if (cudaError_t e = cudaGetLastError()) return (int)e;
    it_done += batch;
  }
  if (iters) *iters = (int)host[S_ITER];
  if (relres) *relres = host[S_RZ] / host[S_RZ0];
  return (int)host[S_STATUS];
}

template <class Op>
static int pcg_fp64(const Op& A, int64_t n, const double* b, double* x, double tol, int max_iter, int check_every,
                    int jacobi, double* work, int32_t* iters, double* relres, cudaStream_t s) {
  PcgWork W = carve(work, n);
  cudaMemsetAsync(W.counter, 0, 2 * sizeof(unsigned), s);
  diag_inv(A, W.dinv, jacobi, s);
  int it = 0;
  int r = pcg_core<Op, double>(A, n, b, x, W.r, W.z, W.p, W.q, W.dinv, W.st, W.counter, W.part, tol, max_iter,
                               check_every, &it, relres, s);
  if (iters) *iters = it;
  return r;
}

// Mixed precision: outer FP64 residual r = b - A x (stop test as above);
// inner FP32 PCG on A32 d = r to `inner_tol`; x += d.
template <class Op64, class Op32>
static int pcg_mixed(const Op64& A, const Op32& A32, int64_t n, const double* b, double* x, double tol,
                     double inner_tol, int max_iter, int check_every, double* work, int32_t* iters, int32_t* outer,
                     double* relres, cudaStream_t s) {
  // FP32 CG with FP64 residual replacement: the FP32 iterate x32 holds the
  // correction since the last replacement; every `check_every` iterations
  // x64 += x32, the true residual b - A x64 is formed in FP64 and replaces
  // the FP32 one, and the recurrence continues with the same search
  // direction.  The stop test is the FP64 one, on the true residual.
  // inner_tol > 0: a batch ends in a replacement only once the FP32
  // recurrence's r.z has fallen below inner_tol times its value at the last
  // replacement (or the FP64 stop test may pass, or it broke down, or the
  // cap is reached); otherwise the FP32 recurrence continues.  inner_tol <= 0
  // replaces after every batch.
  PcgWork W = carve(work, n);                 // st64 and r64 (FP64 residual), dinv
  double* st2 = work + S_LEN + 2 + 5 * n + part_len(n);
  unsigned* counter2 = (unsigned*)(st2 + S_LEN);
  float* f = (float*)(st2 + S_LEN + 2);
  float *xf = f, *rf = f + n, *zf = f + 2 * n, *pf = f + 3 * n, *qf = f + 4 * n;
  cudaMemsetAsync(W.counter, 0, 2 * sizeof(unsigned), s);
  cudaMemsetAsync(counter2, 0, 2 * sizeof(unsigned), s);
  diag_inv(A, W.dinv, 1, s);
  const unsigned vg = vec_grid<double>(n);
  const unsigned vgf = vec_grid<float>(n);
  // FP64 residual of the initial guess and the reference norm b.D^-1 b
  spmv(A, (const double*)x, W.r, nullptr, nullptr, nullptr, 0, s);
  k_pcg_setup<double><<<vg, PCG_TPB, 0, s>>>(n, b, W.r, W.z, W.p, W.dinv, W.st, W.part, W.counter);
  count_launch();
  double h64[S_LEN];
  cudaMemcpyAsync(h64, W.st, sizeof(h64), cudaMemcpyDeviceToHost, s);
  if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
  double rel = h64[S_RZ] / h64[S_RZ0];
  int total = 0, nrep = 0;
  int status = FEA_ENOTCONV;
  if (h64[S_DONE] != 0.0 || rel < tol) {
    status = FEA_OK;
  } else {
    // FP32 start from r64: x32 = 0, r32 = r64, z32, p32, rho; stop test scale from b
    cudaMemsetAsync(xf, 0, sizeof(float) * n, s);
    cudaMemsetAsync(rf, 0, sizeof(float) * n, s);
    k_pcg_setup<float><<<vgf, PCG_TPB, 0, s>>>(n, W.r, rf, zf, pf, W.dinv, st2, W.part, counter2);
    count_launch();
    cudaMemcpyAsync(st2 + S_RZ0, W.st + S_RZ0, sizeof(double), cudaMemcpyDeviceToDevice, s);
    const int ce = std::max(1, check_every);
    double rz_last = h64[S_RZ];
    while (total < max_iter) {
      const int batch = std::min(ce, max_iter - total);
      for (int k = 0; k < batch; ++k) {
        spmv(A32, (const float*)pf, qf, st2, W.part, counter2, 1, s);
        k_pcg_update<float><<<vgf, PCG_TPB, 0, s>>>(n, xf, rf, zf, pf, qf, W.dinv, st2, W.part, counter2, 0.0,
                                                   max_iter);
        count_launch();
        if (k + 1 < batch) {
          k_pcg_p<float><<<vgf, PCG_TPB, 0, s>>>(n, pf, zf, st2);
          count_launch();
        }
      }
      total += batch;
      if (inner_tol > 0.0 && total < max_iter) {
        double h32[S_LEN];
        cudaMemcpyAsync(h32, st2, sizeof(h32), cudaMemcpyDeviceToHost, s);
        if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
        const double rz32 = h32[S_RZ];
        if (h32[S_STATUS] != (double)FEA_EBREAKDOWN && rz32 > inner_tol * rz_last &&
            rz32 / h64[S_RZ0] >= tol) {
          k_pcg_p<float><<<vgf, PCG_TPB, 0, s>>>(n, pf, zf, st2);
          count_launch();
          continue;
        }
      }
      // replacement: x64 += x32, r64 = b - A x64, r32 / z32 / rho / beta from it
      k_axpy_f32<<<grid_for(n, 256), 256, 0, s>>>(n, x, xf);
      cudaMemsetAsync(xf, 0, sizeof(float) * n, s);
      spmv(A, (const double*)x, W.r, nullptr, nullptr, nullptr, 0, s);
      k_mixed_replace<<<vg, PCG_TPB, 0, s>>>(n, b, W.r, W.dinv, rf, zf, W.st, st2, W.part, W.counter, tol);
      k_pcg_p<float><<<vgf, PCG_TPB, 0, s>>>(n, pf, zf, st2);
      count_launch(3);
      ++nrep;
      double h32[S_LEN];
      cudaMemcpyAsync(h64, W.st, sizeof(h64), cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(h32, st2, sizeof(h32), cudaMemcpyDeviceToHost, s);
      if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
      rel = h64[S_RZ] / h64[S_RZ0];
      rz_last = h64[S_RZ];
      if (rel < tol) { status = FEA_OK; break; }
      if (h32[S_STATUS] == (double)FEA_EBREAKDOWN) { status = FEA_EBREAKDOWN; break; }
    }
  }
  if (iters) *iters = total;
  if (outer) *outer = nrep;
  if (relres) *relres = rel;
  return status;
}

template <class V>
static NodeOp<V> node_op(const fea_nodes_t* N, const int32_t* idx, const V* val) {
  return NodeOp<V>{N->vbase_dev, N->rowlen_dev, N->dbase_dev, N->mask_dev, idx, val, N->n_nodes, N->ndof};
}

static bool nodes_ok(const fea_nodes_t* N) {
  return N && N->n_nodes >= 0 && N->ndof >= 0 && (N->ndof == 0 || (N->vbase_dev && N->rowlen_dev && N->dbase_dev &&
                                                                   N->mask_dev));
}

static int read_nnz(const int64_t* ip, int64_t n, int64_t* nnz, cudaStream_t s) {
  *nnz = 0;
  if (cudaError_t e = cudaMemcpyAsync(nnz, ip + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s)) return (int)e;
  return (int)cudaStreamSynchronize(s);
}

// ---- batched PCG over independent systems ("slots") ---------------------
// Work items are warp-sized and a fixed function of the slot alone: SpMV
// items of 16 nodes (plan layout: two nodes at a time per warp, 16 lanes
// each, with the next pair's column indices prefetched) or 16 rows (plain
// CSR), update items of 256 rows.  Each item's warp writes one partial sum
// and counts itself on the slot's counter; the warp that completes the
// slot's count sums the partials in item order and updates the slot's
// scalars.  Warps walk the item lists of all active slots in grid-stride
// order with no block-level barrier.  A slot's arithmetic depends only on
// its own items, so its iterates are the same bits alone or batched.
constexpr int PCGB_ROWS = 256;      // rows per update item and per start chunk
#ifndef FEA_PCGB_GROUP
#define FEA_PCGB_GROUP 16
#endif
constexpr int PCGB_GROUP = FEA_PCGB_GROUP;   // nodes (plan layout) or rows (CSR) per SpMV item

struct PcgbSlotDev {
  const int64_t* ptr;
  const int32_t* idx;
  const double* val;
  const double* b;
  double* x;
  double* st;
  unsigned* counter;       // [0] SpMV items, [1] update items, [2] start chunks
  double *dinv, *r, *z, *p, *q;
  double *part_s, *part_u, *part_0;
  const int64_t* vbase;    // plan layout (node rows), or NULL: plain CSR rows
  const int32_t* rowlen;
  const int32_t* dbase;
  const uint8_t* mask;
  int64_t n, n_nodes;
  int32_t nitem_s, nitem_u, nchunk0, lanes;
  double tol;
  int32_t max_iter, pad;
};

struct PcgbHeader {
  int64_t nitem_s;
  int64_t nitem_u;
  int64_t nslots;
};

struct PcgbView {
  PcgbHeader* hdr;
  PcgbSlotDev* slots;
  int32_t *s_slot, *s_local, *u_slot, *u_local;
};

static PcgbView pcgb_view(void* table, int32_t max_slots, int64_t max_items) {
  PcgbView v;
  char* c = (char*)table;
  v.hdr = (PcgbHeader*)c;
  v.slots = (PcgbSlotDev*)(c + 64);
  v.s_slot = (int32_t*)(c + 64 + sizeof(PcgbSlotDev) * (size_t)max_slots);
  v.s_local = v.s_slot + max_items;
  v.u_slot = v.s_local + max_items;
  v.u_local = v.u_slot + max_items;
  return v;
}

static int64_t pcgb_items_s(int64_t n, int64_t n_nodes) {
  return n_nodes > 0 ? (n_nodes + PCGB_GROUP - 1) / PCGB_GROUP : (n + PCGB_GROUP - 1) / PCGB_GROUP;
}
static int64_t pcgb_items_u(int64_t n) { return (n + PCGB_ROWS - 1) / PCGB_ROWS; }

// A warp that finished `add` items of a slot counts them in the slot's
// completion counter (after a fence that publishes its partial sums) and
// learns whether it completed the slot's last items.
__device__ __forceinline__ bool pcgb_warp_last_n(unsigned* counter, unsigned add, int total, int lane) {
  unsigned old = 0u;
  if (lane == 0) {
    __threadfence();
    old = atomicAdd(counter, add);
  }
  old = __shfl_sync(0xffffffffu, old, 0);
  return old + add == (unsigned)total;
}


__device__ __forceinline__ double pcgb_warp_sum(const double* part, int n, int stride, int off, int lane) {
  // 8 independent L2 loads per lane in flight per batch, fixed order
  double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i0 = 0; i0 < n; i0 += 256) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = i0 + 32 * k + lane;
      v[k] = i < n ? __ldcg(part + (int64_t)i * stride + off) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] += v[k];
  }
  double v = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// q = A p over the node items g0 .. g0 + cnt - 1 of slot S (PCGB_GROUP nodes
// each), two nodes at a time per warp (16 lanes each, 48 columns per pass).
// The next pair's metadata and first-pass column indices are loaded while
// the current pair is processed, across item boundaries, so a run of items
// streams like one long item; each item's p.q is reduced by the same fixed
// tree over the warp and written to part_s[g] when the item ends: an item's
// sums do not depend on the run it is processed in.  (With the register
// count capped for 4 CTAs per SM the kernel ran 24% slower.)
__device__ __forceinline__ void pcgb_nodes_spmv_run(const PcgbSlotDev& S, int g0, int cnt, int lane) {
  const int h = lane >> 4, hl = lane & 15;
  const int64_t nbeg = (int64_t)g0 * PCGB_GROUP;
  const int64_t nend = min((int64_t)(g0 + cnt) * PCGB_GROUP, S.n_nodes);
  double contrib = 0.0;
  int64_t nd = nbeg + h;
  unsigned m = 0;
  int L = 0;
  int64_t vb = 0;
  int32_t jn[3] = {0, 0, 0};
  if (nd < nend) {
    m = S.mask[nd];
    L = m ? S.rowlen[nd] : 0;
    vb = S.vbase[nd];
#pragma unroll
    for (int k = 0; k < 3; ++k) jn[k] = hl + 16 * k < L ? __ldg(S.idx + vb + hl + 16 * k) : 0;
  }
  int g = g0;
  int64_t item_end = min(nbeg + PCGB_GROUP, nend);
  for (int64_t base = nbeg; base < nend; base += 2) {          // warp-uniform
    const int64_t nx = nd + 2;
    unsigned m2 = 0;
    int L2 = 0;
    int64_t vb2 = 0;
    if (nx < nend) {
      m2 = S.mask[nx];
      L2 = S.rowlen[nx];
      vb2 = S.vbase[nx];
    }
    const int f = popc3(m);
    int Lmax = L;
    Lmax = max(Lmax, __shfl_xor_sync(0xffffffffu, Lmax, 16));
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const double* __restrict__ v0 = S.val + vb;
    for (int q0 = 0; q0 < Lmax; q0 += 48) {
      int32_t j[3];
      bool hv[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int q = q0 + hl + 16 * k;
        hv[k] = q < L;
        j[k] = q0 == 0 ? jn[k] : (hv[k] ? __ldg(S.idx + vb + q) : 0);
      }
      double va[3][3];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int q = q0 + hl + 16 * k;
          va[r][k] = (r < f && hv[k]) ? __ldcs(v0 + (int64_t)r * L + q) : 0.0;
        }
      double xv[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) xv[k] = hv[k] ? S.p[j[k]] : 0.0;
      s0 += va[0][0] * xv[0] + va[0][1] * xv[1] + va[0][2] * xv[2];
      s1 += va[1][0] * xv[0] + va[1][1] * xv[1] + va[1][2] * xv[2];
      s2 += va[2][0] * xv[0] + va[2][1] * xv[1] + va[2][2] * xv[2];
    }
    const int Ln = m2 ? L2 : 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) jn[k] = hl + 16 * k < Ln ? __ldg(S.idx + vb2 + hl + 16 * k) : 0;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o, 16);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o, 16);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o, 16);
    }
    if (m && hl < f) {
      const int64_t r = S.dbase[nd] + hl;
      const double sr = hl == 0 ? s0 : (hl == 1 ? s1 : s2);
      S.q[r] = sr;
      contrib += sr * S.p[r];
    }
    nd = nx;
    m = m2;
    L = Ln;
    vb = vb2;
    if (base + 2 >= item_end) {                                 // the item's last pair
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
      if (lane == 0) S.part_s[g] = contrib;
      contrib = 0.0;
      ++g;
      item_end = min(item_end + PCGB_GROUP, nend);
    }
  }
}

// q = A p over CSR rows [r0, r1), LANES lanes per row; returns p.q (lane 0)
template <int LANES>
__device__ __forceinline__ double pcgb_rows_spmv(const PcgbSlotDev& S, int64_t r0, int64_t r1, int lane) {
  constexpr int RPP = 32 / LANES;
  const int sl = lane % LANES, sub = lane / LANES;
  double contrib = 0.0;
  for (int64_t base = r0; base < r1; base += RPP) {
    const int64_t row = base + sub;
    double s = 0.0;
    if (row < r1) {
      const int64_t b = S.ptr[row], e = S.ptr[row + 1];
      for (int64_t i = b + sl; i < e; i += LANES) s += S.val[i] * S.p[S.idx[i]];
    }
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
    if (row < r1 && sl == 0) {
      S.q[row] = s;
      contrib += s * S.p[row];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
  return lane == 0 ? contrib : 0.0;
}

// Each warp takes a contiguous range of the item list (items of one slot are
// consecutive in it) and processes it slot run by slot run: the node-row
// SpMV streams through a run's items without stopping at their boundaries,
// and the slot's completion counter advances once per run.
__global__ void __launch_bounds__(PCG_TPB) k_pcgb_spmv(PcgbView V) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * PCG_WARPS;
  const int64_t nit = V.hdr->nitem_s;
  const int64_t per = (nit + nw - 1) / nw;
  int64_t it = ((int64_t)blockIdx.x * PCG_WARPS + (threadIdx.x >> 5)) * per;
  const int64_t it_end = min(nit, it + per);
  while (it < it_end) {                           // warp-uniform
    const PcgbSlotDev& S = V.slots[V.s_slot[it]];
    const int g0 = V.s_local[it];
    const int cnt = (int)min(it_end - it, (int64_t)S.nitem_s - g0);
    it += cnt;
    if (S.st[S_DONE] != 0.0) continue;
    if (S.vbase) {
      pcgb_nodes_spmv_run(S, g0, cnt, lane);
    } else {
      for (int g = g0; g < g0 + cnt; ++g) {
        const int64_t r0 = (int64_t)g * PCGB_GROUP, r1 = min(r0 + PCGB_GROUP, S.n);
        const double c = S.lanes == 32 ? pcgb_rows_spmv<32>(S, r0, r1, lane)
                                       : (S.lanes == 16 ? pcgb_rows_spmv<16>(S, r0, r1, lane)
                                                        : pcgb_rows_spmv<8>(S, r0, r1, lane));
        if (lane == 0) S.part_s[g] = c;
      }
    }
    if (pcgb_warp_last_n(S.counter + 0, (unsigned)cnt, S.nitem_s, lane)) {
      const double pq = pcgb_warp_sum(S.part_s, S.nitem_s, 1, 0, lane);
      if (lane == 0) {
        S.st[S_PQ] = pq;
        if (!(pq > 0.0) || !isfinite(pq)) {
          S.st[S_STATUS] = (double)FEA_EBREAKDOWN;
          S.st[S_DONE] = 1.0;
          S.st[S_ALPHA] = 0.0;
        } else {
          S.st[S_ALPHA] = S.st[S_RZ] / pq;
        }
        S.counter[0] = 0u;
      }
    }
  }
}

// The vector kernels take contiguous runs of the update item list as the
// SpMV does: the slot's pointers and scalars are read once per run and its
// completion counter advances once per run.
__global__ void __launch_bounds__(PCG_TPB) k_pcgb_update(PcgbView V) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * PCG_WARPS;
  const int64_t nit = V.hdr->nitem_u;
  const int64_t per = (nit + nw - 1) / nw;
  int64_t it = ((int64_t)blockIdx.x * PCG_WARPS + (threadIdx.x >> 5)) * per;
  const int64_t it_end = min(nit, it + per);
  while (it < it_end) {                           // warp-uniform
    const PcgbSlotDev& S = V.slots[V.u_slot[it]];
    const int l0 = V.u_local[it];
    const int cnt = (int)min(it_end - it, (int64_t)S.nitem_u - l0);
    it += cnt;
    if (S.st[S_DONE] != 0.0) continue;
    const double alpha = S.st[S_ALPHA];
    double* __restrict__ x = S.x;
    double* __restrict__ r = S.r;
    double* __restrict__ z = S.z;
    const double* __restrict__ p = S.p;
    const double* __restrict__ q = S.q;
    const double* __restrict__ dinv = S.dinv;
    const int64_t n = S.n;
    for (int l = l0; l < l0 + cnt; ++l) {
      constexpr int K = PCGB_ROWS / 32;
      double xv[K], pv[K], rv[K], qv[K], dv[K];
      const int64_t i0 = (int64_t)l * PCGB_ROWS + lane;
#pragma unroll
      for (int k = 0; k < K; ++k) {            // all loads of the item first
        const int64_t i = i0 + 32 * k;
        const bool in = i < n;
        xv[k] = in ? x[i] : 0.0;
        pv[k] = in ? p[i] : 0.0;
        rv[k] = in ? r[i] : 0.0;
        qv[k] = in ? q[i] : 0.0;
        dv[k] = in ? dinv[i] : 0.0;
      }
      double c = 0.0;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int64_t i = i0 + 32 * k;
        if (i < n) {
          x[i] = xv[k] + alpha * pv[k];
          const double ri = rv[k] - alpha * qv[k];
          r[i] = ri;
          const double zi = ri * dv[k];
          z[i] = zi;
          c += ri * zi;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) S.part_u[l] = c;
    }
    if (pcgb_warp_last_n(S.counter + 1, (unsigned)cnt, S.nitem_u, lane)) {
      const double rz = pcgb_warp_sum(S.part_u, S.nitem_u, 1, 0, lane);
      if (lane == 0) {
        const double iter = S.st[S_ITER] + 1.0;
        S.st[S_ITER] = iter;
        S.st[S_BETA] = rz / S.st[S_RZ];
        S.st[S_RZ] = rz;
        if (!isfinite(rz)) {
          S.st[S_STATUS] = (double)FEA_EBREAKDOWN;
          S.st[S_DONE] = 1.0;
        } else if (rz / S.st[S_RZ0] < S.tol) {
          S.st[S_DONE] = 1.0;
        } else if (iter >= (double)S.max_iter) {
          S.st[S_STATUS] = (double)FEA_ENOTCONV;
          S.st[S_DONE] = 1.0;
        }
        S.counter[1] = 0u;
      }
    }
  }
}

__global__ void __launch_bounds__(PCG_TPB) k_pcgb_p(PcgbView V) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * PCG_WARPS;
  const int64_t nit = V.hdr->nitem_u;
  const int64_t per = (nit + nw - 1) / nw;
  int64_t it = ((int64_t)blockIdx.x * PCG_WARPS + (threadIdx.x >> 5)) * per;
  const int64_t it_end = min(nit, it + per);
  while (it < it_end) {                           // warp-uniform
    const PcgbSlotDev& S = V.slots[V.u_slot[it]];
    const int l0 = V.u_local[it];
    const int cnt = (int)min(it_end - it, (int64_t)S.nitem_u - l0);
    it += cnt;
    if (S.st[S_DONE] != 0.0) continue;
    const double beta = S.st[S_BETA];
    double* __restrict__ p = S.p;
    const double* __restrict__ z = S.z;
    const int64_t n = S.n;
    for (int l = l0; l < l0 + cnt; ++l) {
      constexpr int K = PCGB_ROWS / 32;
      double zv[K], pv[K];
      const int64_t i0 = (int64_t)l * PCGB_ROWS + lane;
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int64_t i = i0 + 32 * k;
        zv[k] = i < n ? z[i] : 0.0;
        pv[k] = i < n ? p[i] : 0.0;
      }
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int64_t i = i0 + 32 * k;
        if (i < n) p[i] = zv[k] + beta * pv[k];
      }
    }
  }
}

// start of one slot: dinv, r = b - A x, z, p, r.z and b.dinv.b; one CTA per
// 256-row chunk (CSR rows: the initial residual is computed once per solve)
template <int LANES>
__device__ __forceinline__ double pcgb_row_ax(const PcgbSlotDev& S, int64_t row, int lane) {
  double s = 0.0;
  if (row < S.n) {
    const int64_t b = S.ptr[row], e = S.ptr[row + 1];
    for (int64_t i = b + lane; i < e; i += LANES) s += S.val[i] * S.x[S.idx[i]];
  }
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
  return s;
}

template <int LANES>
__global__ void __launch_bounds__(PCG_TPB) k_pcgb_start(PcgbView V, int32_t slot) {
  __shared__ double sh[PCG_WARPS];
  static_assert(PCGB_ROWS == PCG_TPB, "the second phase takes one thread per row of the chunk");
  const PcgbSlotDev& S = V.slots[slot];
  // the grid comes from the caller's row count: chunks beyond the slot's own
  // (whose partials would land past its work buffer) leave at once
  if ((int64_t)blockIdx.x >= (int64_t)S.nchunk0) return;
  constexpr int RPP = PCG_TPB / LANES;
  const int lane = threadIdx.x % LANES, sub = threadIdx.x / LANES;
  const int64_t row0 = (int64_t)blockIdx.x * PCGB_ROWS;
  for (int k = 0; k < PCGB_ROWS; k += RPP) {
    const int64_t row = row0 + k + sub;
    const double s = pcgb_row_ax<LANES>(S, row, lane);
    if (row < S.n && lane == 0) S.r[row] = s;
  }
  __syncthreads();
  double c_rz = 0.0, c_bb = 0.0;
  const int64_t i = row0 + threadIdx.x;
  if (i < S.n) {
    int64_t lo = S.ptr[i], hi = S.ptr[i + 1];
    double dv = 0.0;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      const int32_t c = S.idx[mid];
      if (c == i) { dv = S.val[mid]; break; }
      if (c < i) lo = mid + 1; else hi = mid;
    }
    dv = fabs(dv);
    const double di = dv == 0.0 ? 1.0 : 1.0 / dv;
    S.dinv[i] = di;
    const double ri = S.b[i] - S.r[i];
    S.r[i] = ri;
    const double zi = ri * di;
    S.z[i] = zi;
    S.p[i] = zi;
    c_rz = ri * zi;
    c_bb = S.b[i] * S.b[i] * di;
  }
  const double s1 = block_sum_w(c_rz, sh);
  const double s2 = block_sum_w(c_bb, sh);
  if (threadIdx.x == 0) {
    S.part_0[2 * blockIdx.x] = s1;
    S.part_0[2 * blockIdx.x + 1] = s2;
  }
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(S.counter + 2, 1u) == (unsigned)(S.nchunk0 - 1);
  __syncthreads();
  if (last) {
    const double rz = sum_partials(S.part_0, S.nchunk0, 2, 0, sh);
    const double bb = sum_partials(S.part_0, S.nchunk0, 2, 1, sh);
    if (threadIdx.x == 0) {
      S.st[S_RZ] = rz;
      S.st[S_RZ0] = bb == 0.0 ? 1.0 : bb;
      S.st[S_ITER] = 0.0;
      S.st[S_STATUS] = 0.0;
      S.st[S_DONE] = (bb == 0.0 || rz == 0.0 || rz / (bb == 0.0 ? 1.0 : bb) < S.tol || S.max_iter <= 0) ? 1.0 : 0.0;
      S.counter[2] = 0u;
    }
  }
}

// compact per-slot state for the host: done, iterations, status, r.z / b.b
__global__ void k_pcgb_state(PcgbView V, int32_t nslots, double* out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  const double* st = V.slots[s].st;
  if (!st) return;
  out[4 * s + 0] = st[S_DONE];
  out[4 * s + 1] = st[S_ITER];
  out[4 * s + 2] = st[S_STATUS];
  out[4 * s + 3] = st[S_RZ] / st[S_RZ0];
}

}  // namespace fea

using namespace fea;

extern "C" int64_t fea_pcg_work_len(int64_t n) { return S_LEN + 2 + 5 * n + part_len(n); }

extern "C" int64_t fea_pcg_mixed_work_len(int64_t n) {
  // FP64: st | counter | dinv | r | z | p | q | part ; FP32 inner: st2 | counter2 | x,r,z,p,q (floats)
  return fea_pcg_work_len(n) + S_LEN + 2 + (5 * n + 1) / 2;
}

extern "C" int fea_spmv(int64_t n, const int64_t* ip, const int32_t* ix, const double* v, const double* x,
                        double* y, cudaStream_t s) {
  if (n < 0 || !ip || !ix || !v || !x || !y) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  int64_t nnz = 0;
  if (int r = read_nnz(ip, n, &nnz, s)) return r;
  spmv(CsrOp<double>{ip, ix, v, n, nnz}, x, y, nullptr, nullptr, nullptr, 0, s);
  return (int)cudaGetLastError();
}

extern "C" int fea_spmv_nodes(const fea_nodes_t* N, const int32_t* ix, const double* v, const double* x, double* y,
                              cudaStream_t s) {
  if (!nodes_ok(N) || !ix || !v || !x || !y) return FEA_EINVAL;
  if (N->ndof == 0) return FEA_OK;
  spmv(node_op<double>(N, ix, v), x, y, nullptr, nullptr, nullptr, 0, s);
  return (int)cudaGetLastError();
}

extern "C" int fea_convert_f32(int64_t nnz, const double* v, float* v32, cudaStream_t s) {
  if (nnz < 0 || !v || !v32) return FEA_EINVAL;
  if (nnz == 0) return FEA_OK;
  k_f64_to_f32<<<148 * 16, 256, 0, s>>>(nnz, v, v32);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_pcg_solve(int64_t n, const int64_t* ip, const int32_t* ix, const double* v, const double* b,
                             double* x, double tol, int32_t max_iter, int32_t check_every, int32_t jacobi,
                             double* work, int64_t work_len, int32_t* iters, double* relres, cudaStream_t s) {
  if (n < 0 || !ip || !ix || !v || !b || !x || !work || max_iter < 0) return FEA_EINVAL;
  if (work_len < fea_pcg_work_len(n)) return FEA_EWORK;
  if (iters) *iters = 0;
  if (relres) *relres = 0.0;
  if (n == 0) return FEA_OK;
  int64_t nnz = 0;
  if (int r = read_nnz(ip, n, &nnz, s)) return r;
  return pcg_fp64(CsrOp<double>{ip, ix, v, n, nnz}, n, b, x, tol, max_iter, check_every, jacobi, work, iters,
                  relres, s);
}

extern "C" int fea_pcg_solve_nodes(const fea_nodes_t* N, const int32_t* ix, const double* v, const double* b,
                                   double* x, double tol, int32_t max_iter, int32_t check_every, double* work,
                                   int64_t work_len, int32_t* iters, double* relres, cudaStream_t s) {
  if (!nodes_ok(N) || !ix || !v || !b || !x || !work || max_iter < 0) return FEA_EINVAL;
  const int64_t n = N->ndof;
  if (work_len < fea_pcg_work_len(n)) return FEA_EWORK;
  if (iters) *iters = 0;
  if (relres) *relres = 0.0;
  if (n == 0) return FEA_OK;
  return pcg_fp64(node_op<double>(N, ix, v), n, b, x, tol, max_iter, check_every, 1, work, iters, relres, s);
}

extern "C" int fea_pcg_solve_mixed(int64_t n, const int64_t* ip, const int32_t* ix, const double* v,
                                   const float* v32, const double* b, double* x, double tol, double inner_tol,
                                   int32_t max_iter, int32_t check_every, double* work, int64_t work_len,
                                   int32_t* iters, int32_t* outer, double* relres, cudaStream_t s) {
  if (n < 0 || !ip || !ix || !v || !v32 || !b || !x || !work || max_iter < 0) return FEA_EINVAL;
  if (work_len < fea_pcg_mixed_work_len(n)) return FEA_EWORK;
  if (iters) *iters = 0;
  if (outer) *outer = 0;
  if (relres) *relres = 0.0;
  if (n == 0) return FEA_OK;
  int64_t nnz = 0;
  if (int r = read_nnz(ip, n, &nnz, s)) return r;
  return pcg_mixed(CsrOp<double>{ip, ix, v, n, nnz}, CsrOp<float>{ip, ix, v32, n, nnz}, n, b, x, tol, inner_tol,
                   max_iter, check_every, work, iters, outer, relres, s);
}

extern "C" int fea_pcg_solve_mixed_nodes(const fea_nodes_t* N, const int32_t* ix, const double* v, const float* v32,
                                         const double* b, double* x, double tol, double inner_tol, int32_t max_iter,
                                         int32_t check_every, double* work, int64_t work_len, int32_t* iters,
                                         int32_t* outer, double* relres, cudaStream_t s) {
  if (!nodes_ok(N) || !ix || !v || !v32 || !b || !x || !work || max_iter < 0) return FEA_EINVAL;
  const int64_t n = N->ndof;
  if (work_len < fea_pcg_mixed_work_len(n)) return FEA_EWORK;
  if (iters) *iters = 0;
  if (outer) *outer = 0;
  if (relres) *relres = 0.0;
  if (n == 0) return FEA_OK;
  return pcg_mixed(node_op<double>(N, ix, v), node_op<float>(N, ix, v32), n, b, x, tol, inner_tol, max_iter,
                   check_every, work, iters, outer, relres, s);
}

static bool layout_ok(const fea_f32_layout_t* Q) {
  return Q && Q->cbase_dev && Q->qbase_dev && Q->cols_dev && Q->vals_dev;
}

extern "C" int fea_f32_layout_fill(const fea_nodes_t* N, const int32_t* ix, const double* v, fea_f32_layout_t* Q,
                                   int32_t with_cols, cudaStream_t s) {
  if (!nodes_ok(N) || !ix || !v || !layout_ok(Q)) return FEA_EINVAL;
  if (N->n_nodes == 0) return FEA_OK;
  const unsigned grid = (unsigned)((N->n_nodes * 32 + 255) / 256);
  k_fill_node32q<<<grid, 256, 0, s>>>(node_op<double>(N, ix, v), Q->cbase_dev, Q->qbase_dev,
                                      with_cols ? Q->cols_dev : nullptr, Q->vals_dev);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_pcg_solve_mixed_nodes32(const fea_nodes_t* N, const int32_t* ix, const double* v,
                                           const fea_f32_layout_t* Q, const double* b, double* x, double tol,
                                           double inner_tol, int32_t max_iter, int32_t check_every, double* work,
                                           int64_t work_len, int32_t* iters, int32_t* outer, double* relres,
                                           cudaStream_t s) {
  if (!nodes_ok(N) || !ix || !v || !layout_ok(Q) || !b || !x || !work || max_iter < 0) return FEA_EINVAL;
  const int64_t n = N->ndof;
  if (work_len < fea_pcg_mixed_work_len(n)) return FEA_EWORK;
  if (iters) *iters = 0;
  if (outer) *outer = 0;
  if (relres) *relres = 0.0;
  if (n == 0) return FEA_OK;
  const NodeOp32q A32{Q->cbase_dev, Q->qbase_dev, Q->cols_dev, Q->vals_dev, N->mask_dev, N->dbase_dev,
                      N->n_nodes, n};
  return pcg_mixed(node_op<double>(N, ix, v), A32, n, b, x, tol, inner_tol, max_iter, check_every, work, iters,
                   outer, relres, s);
}

// ---- batched PCG C ABI ------------------------------------------------------
extern "C" int64_t fea_pcgb_work_len(int64_t n, int64_t n_nodes) {
  return S_LEN + 2 + 5 * n + pcgb_items_s(n, n_nodes) + pcgb_items_u(n) + 2 * pcgb_items_u(n) + 2;
}

extern "C" int64_t fea_pcgb_table_bytes(int32_t max_slots, int64_t max_items) {
  if (max_slots <= 0 || max_items <= 0) return 0;
  return 64 + (int64_t)sizeof(PcgbSlotDev) * max_slots + 16 * max_items;
}

extern "C" int fea_pcgb_set(void* table, int32_t max_slots, int64_t max_items, int32_t nslots,
                            const fea_pcgb_slot_t* slots, cudaStream_t s) {
  if (!table || max_slots <= 0 || max_items <= 0 || nslots < 0 || nslots > max_slots || (nslots && !slots))
    return FEA_EINVAL;
  std::vector<PcgbSlotDev> dev(nslots);
  std::vector<int32_t> ss, sl, us, ul;
  for (int32_t k = 0; k < nslots; ++k) {
    const fea_pcgb_slot_t& h = slots[k];
    PcgbSlotDev& d = dev[k];
    std::memset(&d, 0, sizeof(d));
    if (h.n < 0 || h.n_nodes < 0) return FEA_EINVAL;
    if (!h.work_dev) continue;                       // empty slot
    if (h.n > 0 && (!h.indptr_dev || !h.indices_dev || !h.values_dev || !h.b_dev || !h.x_dev)) return FEA_EINVAL;
    const int64_t nn = h.vbase_dev ? h.n_nodes : 0;
    if (h.vbase_dev && (!h.rowlen_dev || !h.dbase_dev || !h.mask_dev)) return FEA_EINVAL;
    if (h.work_len < fea_pcgb_work_len(h.n, nn)) return FEA_EWORK;
    const int64_t is = pcgb_items_s(h.n, nn), iu = pcgb_items_u(h.n);
    if (is >= INT32_MAX || iu >= INT32_MAX) return FEA_ERANGE;
    double* w = h.work_dev;
    d.ptr = h.indptr_dev; d.idx = h.indices_dev; d.val = h.values_dev; d.b = h.b_dev; d.x = h.x_dev;
    d.st = w;
    d.counter = (unsigned*)(w + S_LEN);
    d.dinv = w + S_LEN + 2;
    d.r = d.dinv + h.n; d.z = d.r + h.n; d.p = d.z + h.n; d.q = d.p + h.n;
    d.part_s = d.q + h.n; d.part_u = d.part_s + is; d.part_0 = d.part_u + iu;
    if (h.vbase_dev) { d.vbase = h.vbase_dev; d.rowlen = h.rowlen_dev; d.dbase = h.dbase_dev; d.mask = h.mask_dev; }
    d.n = h.n;
    d.n_nodes = nn;
    d.nitem_s = (int32_t)is;
    d.nitem_u = (int32_t)iu;
    d.nchunk0 = (int32_t)iu;
    d.lanes = (h.n > 0 && h.nnz > 0) ? lanes_for(h.n, h.nnz) : 8;
    d.tol = h.tol;
    d.max_iter = h.max_iter;
    if (h.active) {
      for (int32_t c = 0; c < d.nitem_s; ++c) { ss.push_back(k); sl.push_back(c); }
      for (int32_t c = 0; c < d.nitem_u; ++c) { us.push_back(k); ul.push_back(c); }
    }
  }
  if ((int64_t)ss.size() > max_items || (int64_t)us.size() > max_items) return FEA_ERANGE;
  // all slots checked: a rejected call has touched no device memory
  for (int32_t k = 0; k < nslots; ++k) {
    // completion counters are zero between kernels; a new work buffer starts so
    if (dev[k].counter)
      if (cudaError_t e = cudaMemsetAsync(dev[k].counter, 0, 4 * sizeof(unsigned), s)) return (int)e;
  }
  PcgbView V = pcgb_view(table, max_slots, max_items);
  PcgbHeader hdr{(int64_t)ss.size(), (int64_t)us.size(), (int64_t)nslots};
  if (cudaError_t e = cudaMemcpyAsync(V.hdr, &hdr, sizeof(hdr), cudaMemcpyHostToDevice, s)) return (int)e;
  if (nslots)
    if (cudaError_t e = cudaMemcpyAsync(V.slots, dev.data(), sizeof(PcgbSlotDev) * nslots, cudaMemcpyHostToDevice, s))
      return (int)e;
  auto put = [&](int32_t* dst, const std::vector<int32_t>& v) -> int {
    if (v.empty()) return 0;
    return (int)cudaMemcpyAsync(dst, v.data(), 4 * v.size(), cudaMemcpyHostToDevice, s);
  };
  if (int r = put(V.s_slot, ss)) return r;
  if (int r = put(V.s_local, sl)) return r;
  if (int r = put(V.u_slot, us)) return r;
  if (int r = put(V.u_local, ul)) return r;
  // the host vectors above are released on return: finish the copies first
  return (int)cudaStreamSynchronize(s);
}

extern "C" int fea_pcgb_start(void* table, int32_t max_slots, int64_t max_items, int32_t slot, int64_t n,
                              int64_t nnz, cudaStream_t s) {
  if (!table || slot < 0 || slot >= max_slots || n < 0 || max_items <= 0) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  PcgbView V = pcgb_view(table, max_slots, max_items);
  const int L = lanes_for(n, nnz);
  const unsigned grid = (unsigned)pcgb_items_u(n);
  if (L == 32) k_pcgb_start<32><<<grid, PCG_TPB, 0, s>>>(V, slot);
  else if (L == 16) k_pcgb_start<16><<<grid, PCG_TPB, 0, s>>>(V, slot);
  else k_pcgb_start<8><<<grid, PCG_TPB, 0, s>>>(V, slot);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_pcgb_iterate(void* table, int32_t max_slots, int64_t max_items, int32_t iters, cudaStream_t s) {
  if (!table || max_slots <= 0 || max_items <= 0 || iters < 0) return FEA_EINVAL;
  PcgbView V = pcgb_view(table, max_slots, max_items);
  const int64_t warps_needed = max_items;
  const unsigned g1 = occ_grid(k_pcgb_spmv, warps_needed, PCG_WARPS);
  const unsigned g2 = occ_grid(k_pcgb_update, warps_needed, PCG_WARPS);
  const unsigned g3 = occ_grid(k_pcgb_p, warps_needed, PCG_WARPS);
  for (int32_t k = 0; k < iters; ++k) {
    k_pcgb_spmv<<<g1, PCG_TPB, 0, s>>>(V);
    k_pcgb_update<<<g2, PCG_TPB, 0, s>>>(V);
    k_pcgb_p<<<g3, PCG_TPB, 0, s>>>(V);
    count_launch(3);
  }
  return (int)cudaGetLastError();
}

extern "C" int fea_pcgb_state(void* table, int32_t max_slots, int64_t max_items, int32_t nslots, double* out_dev,
                              cudaStream_t s) {
  if (!table || nslots < 0 || nslots > max_slots || max_items <= 0 || (nslots && !out_dev)) return FEA_EINVAL;
  if (!nslots) return FEA_OK;
  PcgbView V = pcgb_view(table, max_slots, max_items);
  k_pcgb_state<<<(nslots + 127) / 128, 128, 0, s>>>(V, nslots, out_dev);
  count_launch();
  return (int)cudaGetLastError();
}
