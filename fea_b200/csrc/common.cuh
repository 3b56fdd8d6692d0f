// Shared device helpers for the fea_b200 kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <atomic>
#include <cmath>
#include <mutex>

#include "../../include/fea_b200.h"

namespace fea {

// host-side launch counter (instrumentation only)
void count_launch(int n = 1);

// Reference-element tables, filled once per process from the host.
//   c_dxi_tet[b][m]     dN_b/dxi_m of the linear tet (constant)
//   c_dxi_hex[g][b][m]  dN_b/dxi_m of the trilinear hex at Gauss point g
//   c_N_hex[g][b]       N_b at Gauss point g (mass)
// Surface rules (T3: 3 points, Q4: 4 points):
//   c_sf_t3[g][m][a]    m = 0: N_a, m = 1,2: dN_a/dxi_{m-1}; c_w_t3[g]
//   c_sf_q4[g][m][a]    same for Q4;                          c_w_q4[g]
static __constant__ double c_dxi_tet[4][3];
static __constant__ double c_dxi_hex[8][8][3];
static __constant__ double c_N_hex[8][8];
static __constant__ double c_sf_t3[3][3][3];
static __constant__ double c_w_t3[3];
static __constant__ double c_sf_q4[4][3][4];
static __constant__ double c_w_q4[4];

// Per translation unit: one bit per device whose tables are uploaded.  The
// first call on a device uploads them with synchronous copies under a mutex
// (host threads making their first calls at once wait for one upload), so
// that first call should come before any stream capture on that device.
static std::atomic<unsigned long long> g_tables_ready{0};
static std::mutex g_tables_mu;

static inline int ensure_tables() {
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return (int)err;
  if (dev < 64 && (g_tables_ready.load(std::memory_order_acquire) >> dev & 1ull)) return 0;
  std::lock_guard<std::mutex> lock(g_tables_mu);
  if (dev < 64 && (g_tables_ready.load(std::memory_order_acquire) >> dev & 1ull)) return 0;
  double tet[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const double s[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                          {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double q = 1.0 / std::sqrt(3.0);
  double dhex[8][8][3], Nhex[8][8];
  for (int g = 0; g < 8; ++g)
    for (int b = 0; b < 8; ++b) {
      double f[3];
      for (int m = 0; m < 3; ++m) f[m] = 1.0 + s[b][m] * s[g][m] * q;
      Nhex[g][b] = 0.125 * f[0] * f[1] * f[2];
      dhex[g][b][0] = 0.125 * s[b][0] * f[1] * f[2];
      dhex[g][b][1] = 0.125 * s[b][1] * f[0] * f[2];
      dhex[g][b][2] = 0.125 * s[b][2] * f[0] * f[1];
    }
  // T3: 3-point rule, Q4: 2x2 Gauss (surfaces/triangle.py, quadrilateral.py)
  const double pt3[3][2] = {{1.0 / 6, 1.0 / 6}, {2.0 / 3, 1.0 / 6}, {1.0 / 6, 2.0 / 3}};
  double sf3[3][3][3], w3[3];
  for (int g = 0; g < 3; ++g) {
    double x = pt3[g][0], y = pt3[g][1];
    sf3[g][0][0] = 1 - x - y; sf3[g][0][1] = x; sf3[g][0][2] = y;
    sf3[g][1][0] = -1; sf3[g][1][1] = 1; sf3[g][1][2] = 0;
    sf3[g][2][0] = -1; sf3[g][2][1] = 0; sf3[g][2][2] = 1;
    w3[g] = 1.0 / 6.0;
  }
  const double c4[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  double sf4[4][3][4], w4[4];
  for (int g = 0; g < 4; ++g) {
    double x = c4[g][0] * q, y = c4[g][1] * q;
    for (int a = 0; a < 4; ++a) {
      double fx = 1 + c4[a][0] * x, fy = 1 + c4[a][1] * y;
      sf4[g][0][a] = 0.25 * fx * fy;
      sf4[g][1][a] = 0.25 * c4[a][0] * fy;
      sf4[g][2][a] = 0.25 * c4[a][1] * fx;
    }
    w4[g] = 1.0;
  }
  if ((err = cudaMemcpyToSymbol(c_dxi_tet, tet, sizeof(tet))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_dxi_hex, dhex, sizeof(dhex))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_N_hex, Nhex, sizeof(Nhex))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_sf_t3, sf3, sizeof(sf3))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_w_t3, w3, sizeof(w3))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_sf_q4, sf4, sizeof(sf4))) != cudaSuccess) return (int)err;
  if ((err = cudaMemcpyToSymbol(c_w_q4, w4, sizeof(w4))) != cudaSuccess) return (int)err;
  if (dev < 64) g_tables_ready.fetch_or(1ull << dev, std::memory_order_release);
  return 0;
}


template <int NN>
struct Elem;
template <>
struct Elem<4> {
  static constexpr int NG = 1;
  __device__ static __forceinline__ double dxi(int g, int b, int m) { return c_dxi_tet[b][m]; }
  __device__ static __forceinline__ double wq(int g) { return 1.0 / 6.0; }
  __device__ static __forceinline__ double N(int g, int b) { return 0.25; }
};
template <>
struct Elem<8> {
  static constexpr int NG = 8;
  __device__ static __forceinline__ double dxi(int g, int b, int m) { return c_dxi_hex[g][b][m]; }
  __device__ static __forceinline__ double wq(int g) { return 1.0; }
  __device__ static __forceinline__ double N(int g, int b) { return c_N_hex[g][b]; }
};

// ---- 3x3 (row-major m[3*r+c]) --------------------------------------------
// J^(-2/3) of the Neo-Hookean isochoric part from the reciprocal cube root
// (CUDA's rcbrt, 1 ulp) squared: one special function instead of a general
// power.  J < 0 gives NaN and J = 0 gives +inf, as pow(J, -2/3) does.
__device__ __forceinline__ double jm23(double J) {
  const double r = rcbrt(J);
  return J < 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : r * r;
}

template <class T>
__device__ __forceinline__ T det3(const T m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}
// inverse by the adjugate; returns the determinant
template <class T>
__device__ __forceinline__ T inv3(const T m[9], T r[9]) {
  T c00 = m[4] * m[8] - m[5] * m[7];
  T c01 = m[5] * m[6] - m[3] * m[8];
  T c02 = m[3] * m[7] - m[4] * m[6];
  T d = m[0] * c00 + m[1] * c01 + m[2] * c02;
  T id = T(1) / d;
  r[0] = c00 * id;
  r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c01 * id;
  r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c02 * id;
  r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return d;
}

// Inverse of the deformation gradient with J^(-2/3) from one reciprocal cube
// root r = rcbrt(J): 1/J = r^3 replaces the division of inv3.  Returns J;
// *jm = J^(-2/3) (NaN for J < 0, as pow gives).
__device__ __forceinline__ double inv3_jm(const double m[9], double r[9], double* jm) {
  const double c00 = m[4] * m[8] - m[5] * m[7];
  const double c01 = m[5] * m[6] - m[3] * m[8];
  const double c02 = m[3] * m[7] - m[4] * m[6];
  const double d = m[0] * c00 + m[1] * c01 + m[2] * c02;
  const double cr = rcbrt(d);
  const double id = cr * cr * cr;
  *jm = d < 0.0 ? __longlong_as_double(0x7ff8000000000000LL) : cr * cr;
  r[0] = c00 * id;
  r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c01 * id;
  r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c02 * id;
  r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return d;
}

__device__ __forceinline__ int popc3(unsigned m) { return __popc(m & 7u); }
__device__ __forceinline__ int rank3(unsigned m, int k) { return __popc(m & ((1u << k) - 1u)); }

// displacement component k of node c from the reduced vector
template <class T>
__device__ __forceinline__ T node_u(const T* __restrict__ gc, int32_t rd, unsigned m, int k) {
  return (m >> k & 1u) ? gc[rd + rank3(m, k)] : T(0);
}

// deterministic block sum (power-of-two block size)
template <int BS>
__device__ __forceinline__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
#pragma unroll
  for (int s = BS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}

inline int grid_for(int64_t n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace fea
