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
// partials, summed by the last block to finish), so results are bitwise
// reproducible.  The host reads the status every `check_every` iterations.
#include <cmath>

#include "common.cuh"

namespace fea {

constexpr int PCG_TPB = 256;

// device-side solver state (doubles, in the work buffer)
enum { S_RZ = 0, S_RZ0, S_ALPHA, S_BETA, S_DONE, S_ITER, S_STATUS, S_PQ, S_COUNT, S_LEN = 16 };

template <class V>
struct CsrT {
  const int64_t* __restrict__ ptr;
  const int32_t* __restrict__ idx;
  const V* __restrict__ val;
};

// group of LANES threads per row: dot(row, x)
template <int LANES, class V, class X>
__device__ __forceinline__ double row_dot(const CsrT<V>& A, int64_t row, int64_t n, const X* __restrict__ x,
                                          int lane) {
  double s = 0.0;
  if (row < n) {
    const int64_t b = A.ptr[row], e = A.ptr[row + 1];
    for (int64_t i = b + lane; i < e; i += LANES) s += (double)A.val[i] * (double)x[A.idx[i]];
  }
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, LANES);
  return s;
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

__device__ __forceinline__ double sum_partials(const volatile double* part, int n, double* sh) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += PCG_TPB) acc += part[i];
  return block_sum<PCG_TPB>(acc, sh);
}

// y = A x ; optionally partial dot(x, y) per block -> part
template <int LANES, class V, class X>
__global__ void __launch_bounds__(PCG_TPB) k_spmv_dot(CsrT<V> A, int64_t n, const X* __restrict__ x,
                                                      X* __restrict__ y, double* st, double* part,
                                                      unsigned* counter, int mode) {
  // mode 0: plain y = Ax.  mode 1: PCG step 1 (alpha = rz / p.q).
  __shared__ double sh[PCG_TPB];
  if (mode == 1 && st[S_DONE] != 0.0) return;
  const int groups = PCG_TPB / LANES;
  const int lane = threadIdx.x % LANES;
  const int64_t row = (int64_t)blockIdx.x * groups + threadIdx.x / LANES;
  double contrib = 0.0;
  const double s = row_dot<LANES>(A, row, n, x, lane);   // every lane takes part in the shuffles
  if (row < n && lane == 0) {
    y[row] = (X)s;
    contrib = s * (double)x[row];
  }
  if (mode == 0) return;
  double bs = block_sum<PCG_TPB>(contrib, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
  if (last_block(counter)) {
    double pq = sum_partials(part, gridDim.x, sh);
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

// x += alpha p; r -= alpha q; z = r / |d|; partial r.z; last block: beta, stop test
template <class X>
__global__ void __launch_bounds__(PCG_TPB) k_pcg_update(int64_t n, X* __restrict__ x, X* __restrict__ r,
                                                        X* __restrict__ z, const X* __restrict__ p,
                                                        const X* __restrict__ q, const double* __restrict__ dinv,
                                                        double* st, double* part, unsigned* counter, double tol,
                                                        int max_iter) {
  __shared__ double sh[PCG_TPB];
  if (st[S_DONE] != 0.0) return;
  const double alpha = st[S_ALPHA];
  double contrib = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * PCG_TPB) {
    x[i] = (X)((double)x[i] + alpha * (double)p[i]);
    double ri = (double)r[i] - alpha * (double)q[i];
    r[i] = (X)ri;
    double zi = ri * dinv[i];
    z[i] = (X)zi;
    contrib += ri * zi;
  }
  double bs = block_sum<PCG_TPB>(contrib, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
  if (last_block(counter)) {
    double rz = sum_partials(part, gridDim.x, sh);
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
  for (int64_t i = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * PCG_TPB)
    p[i] = (X)((double)z[i] + beta * (double)p[i]);
}

// setup: dinv = 1/|diag| (0 -> 1), r = b - Ax (Ax in r on entry), z = dinv r,
// p = z, partial r.z and b.dinv.b; last block initialises the state.
template <class X>
__global__ void __launch_bounds__(PCG_TPB) k_pcg_setup(CsrT<double> A, int64_t n, const double* __restrict__ b,
                                                       X* __restrict__ r, X* __restrict__ z, X* __restrict__ p,
                                                       double* __restrict__ dinv, double* st, double* part,
                                                       unsigned* counter, int compute_dinv, double tol) {
  __shared__ double sh[PCG_TPB];
  double c_rz = 0.0, c_bb = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * PCG_TPB + threadIdx.x; i < n; i += (int64_t)gridDim.x * PCG_TPB) {
    double di;
    if (compute_dinv) {
      // diagonal entry: binary search for column i in row i
      int64_t lo = A.ptr[i], hi = A.ptr[i + 1];
      double dv = 0.0;
      while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        int32_t c = A.idx[mid];
        if (c == i) { dv = A.val[mid]; break; }
        if (c < i) lo = mid + 1; else hi = mid;
      }
      dv = fabs(dv);
      di = (compute_dinv == 2 || dv == 0.0) ? 1.0 : 1.0 / dv;
      dinv[i] = di;
    } else {
      di = dinv[i];
    }
    double ri = b[i] - (double)r[i];
    r[i] = (X)ri;
    double zi = ri * di;
    z[i] = (X)zi;
    p[i] = (X)zi;
    c_rz += ri * zi;
    c_bb += b[i] * b[i] * di;
  }
  double s1 = block_sum<PCG_TPB>(c_rz, sh);
  double s2 = block_sum<PCG_TPB>(c_bb, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s1;
    part[2 * blockIdx.x + 1] = s2;
  }
  if (last_block(counter)) {
    double a1 = 0.0, a2 = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += PCG_TPB) {
      a1 += ((volatile double*)part)[2 * i];
      a2 += ((volatile double*)part)[2 * i + 1];
    }
    double rz = block_sum<PCG_TPB>(a1, sh);
    double bb = block_sum<PCG_TPB>(a2, sh);
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

template <class X>
__global__ void k_copy_cast(int64_t n, const double* __restrict__ a, X* __restrict__ b) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (X)a[i];
}

__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

__global__ void k_axpy_f32(int64_t n, double* __restrict__ x, const float* __restrict__ d) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += (double)d[i];
}

static int lanes_for(int64_t n, int64_t nnz) {
  double avg = n ? (double)nnz / (double)n : 0.0;
  return avg >= 40.0 ? 32 : (avg >= 12.0 ? 16 : 8);
}

template <class V, class X>
static void spmv_launch(const CsrT<V>& A, int64_t n, int64_t nnz, const X* x, X* y, double* st, double* part,
                        unsigned* counter, int mode, cudaStream_t s) {
  const int L = lanes_for(n, nnz);
  const int rows_per_block = PCG_TPB / L;
  const unsigned grid = (unsigned)((n + rows_per_block - 1) / rows_per_block);
  if (L == 32) k_spmv_dot<32, V, X><<<grid, PCG_TPB, 0, s>>>(A, n, x, y, st, part, counter, mode);
  else if (L == 16) k_spmv_dot<16, V, X><<<grid, PCG_TPB, 0, s>>>(A, n, x, y, st, part, counter, mode);
  else k_spmv_dot<8, V, X><<<grid, PCG_TPB, 0, s>>>(A, n, x, y, st, part, counter, mode);
  count_launch();
}

static unsigned vec_grid(int64_t n) {
  int64_t g = (n + PCG_TPB - 1) / PCG_TPB;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 8));
}

static int64_t part_len(int64_t n) {
  // partials of the SpMV grid (>= 1 row per 32 threads) and of the vector grid
  return std::max<int64_t>((n + 7) / 8 + 1, 2 * 148 * 8 + 2);
}

// Work layout (doubles): st[S_LEN] | counter(1) | dinv[n] | r | z | p | q | part
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
// dinv given.  Returns status; *iters.
template <class V, class X>
static int pcg_core(const CsrT<V>& A, const CsrT<double>& A64, int64_t n, int64_t nnz, const double* b, X* x,
                    X* r, X* z, X* p, X* q, double* dinv, double* st, unsigned* counter, double* part,
                    int compute_dinv, double tol, int max_iter, int check_every, int* iters, double* relres,
                    cudaStream_t s) {
  // r = A x  (in the working precision), then setup
  spmv_launch<V, X>(A, n, nnz, x, r, st, part, counter, 0, s);
  const unsigned vg = vec_grid(n);
  k_pcg_setup<X><<<vg, PCG_TPB, 0, s>>>(A64, n, b, r, z, p, dinv, st, part, counter, compute_dinv, tol);
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
      spmv_launch<V, X>(A, n, nnz, p, q, st, part, counter, 1, s);
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

}  // namespace fea

using namespace fea;

extern "C" int64_t fea_pcg_work_len(int64_t n) { return S_LEN + 2 + 5 * n + part_len(n); }

extern "C" int fea_spmv(int64_t n, const int64_t* ip, const int32_t* ix, const double* v, const double* x,
                        double* y, cudaStream_t s) {
  if (n < 0 || !ip || !ix || !v || !x || !y) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  int64_t nnz = 0;
  cudaMemcpy(&nnz, ip + n, sizeof(int64_t), cudaMemcpyDeviceToHost);
  CsrT<double> A{ip, ix, v};
  spmv_launch<double, double>(A, n, nnz, x, y, nullptr, nullptr, nullptr, 0, s);
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
  if (cudaError_t e = cudaMemcpyAsync(&nnz, ip + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s)) return (int)e;
  if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
  PcgWork W = carve(work, n);
  cudaMemsetAsync(W.counter, 0, sizeof(unsigned), s);
  CsrT<double> A{ip, ix, v};
  int it = 0;
  int r = pcg_core<double, double>(A, A, n, nnz, b, x, W.r, W.z, W.p, W.q, W.dinv, W.st, W.counter, W.part,
                                   jacobi ? 1 : 2, tol, max_iter, check_every, &it, relres, s);
  if (iters) *iters = it;
  return r;
}

// Mixed precision: outer FP64 residual r = b - A x (stop test as above);
// inner FP32 PCG on A32 d = r to `inner_tol`; x += d.
extern "C" int64_t fea_pcg_mixed_work_len(int64_t n) {
  // FP64 outer: st | counter | dinv | r64 | part ; FP32 inner: x,r,z,p,q (floats) + st2
  return fea_pcg_work_len(n) + (5 * n + 1) / 2 + S_LEN + 2;
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
  if (cudaError_t e = cudaMemcpyAsync(&nnz, ip + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s)) return (int)e;
  if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
  PcgWork W = carve(work, n);                 // r = FP64 residual, q = FP64 A x
  double* st2 = work + fea_pcg_work_len(n);
  unsigned* counter2 = (unsigned*)(st2 + S_LEN);
  float* f = (float*)(st2 + S_LEN + 2);
  float *xf = f, *rf = f + n, *zf = f + 2 * n, *pf = f + 3 * n, *qf = f + 4 * n;
  cudaMemsetAsync(W.counter, 0, sizeof(unsigned), s);
  cudaMemsetAsync(counter2, 0, sizeof(unsigned), s);
  CsrT<double> A{ip, ix, v};
  CsrT<float> A32{ip, ix, v32};
  const unsigned vg = vec_grid(n);
  int total = 0, nouter = 0;
  double rel = 0.0;
  int status = FEA_ENOTCONV;
  bool first = true;
  while (total < max_iter) {
    // FP64 residual, stop test, and the inner right-hand side rf = r
    spmv_launch<double, double>(A, n, nnz, x, W.r, nullptr, nullptr, nullptr, 0, s);
    k_pcg_setup<double><<<vg, PCG_TPB, 0, s>>>(A, n, b, W.r, W.z, W.p, W.dinv, W.st, W.part, W.counter,
                                               first ? 1 : 0, tol);
    count_launch();
    first = false;
    double host[S_LEN];
    cudaMemcpyAsync(host, W.st, sizeof(host), cudaMemcpyDeviceToHost, s);
    if (cudaError_t e = cudaStreamSynchronize(s)) return (int)e;
    rel = host[S_RZ] / host[S_RZ0];
    if (host[S_DONE] != 0.0 || rel < tol) {
      status = FEA_OK;
      break;
    }
    // inner solve: b_inner = r (FP64 in W.r), x_inner = 0
    cudaMemsetAsync(xf, 0, sizeof(float) * n, s);
    int it = 0;
    double rr = 0.0;
    int ri = pcg_core<float, float>(A32, A, n, nnz, W.r, xf, rf, zf, pf, qf, W.dinv, st2, counter2, W.part, 0,
                                    inner_tol, max_iter - total, check_every, &it, &rr, s);
    total += it;
    ++nouter;
    k_axpy_f32<<<grid_for(n, 256), 256, 0, s>>>(n, x, xf);
    count_launch();
    if (ri == FEA_EBREAKDOWN) { status = ri; break; }
    if (it == 0) { status = FEA_EBREAKDOWN; break; }
  }
  if (iters) *iters = total;
  if (outer) *outer = nouter;
  if (relres) *relres = rel;
  return status;
}
