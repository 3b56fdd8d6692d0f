// Adjoint sensitivities of the Neo-Hookean element residual and of the
// follower pressure (sm_100a, FP64).
//
// For an adjoint field lam, Phi = sum_e lam_e . R_e(u, X, mu) with
// R_e[a] = sum_g w P(F) g_a (Element_3D.structural_Force, FEA =
// sssnnn7119/FEA, FEA/assemble/elements/C3/C3base.py:413-452).  Perturbing
// the reference coordinates by dX gives D = sum_b dX_b (x) g_b and
//   dw = w tr D,  dg_a = -D^T g_a,  dF = -(F - I) D,  dLam = -Lam D
// (Lam = sum_a lam_a (x) g_a), so that
//   dPhi/dX_b = sum_g w M g_b,
//   M = (P : Lam) I - (F - I)^T A[Lam] - Lam^T P,
// where A[Lam] = dP/dF[Lam] is the Neo-Hookean tangent applied to Lam
// (materials/hyperelastic.py:69-82, factored: A[Lam]^T = T1 tr(F^-1 Lam) +
// T2 (F : Lam) + T3 Lam F^-1 + mu J^-2/3 Lam^T), and
//   dPhi/dmu = sum_g w (J^-2/3 F - I1/3 F^-T) : Lam.
// The pressure term lam . (p dV/dx) depends on X only through x = X + u, so
// its X-derivative is the Hessian-vector product p d2V/dx2 lam of the
// enclosed-volume functional (loads/pressure.py:80-132).
#include <cmath>

#include "common.cuh"

namespace fea {

struct AdjParams {
  const double* __restrict__ X;
  const int32_t* __restrict__ rdof;
  const uint8_t* __restrict__ mask;
  const int32_t* __restrict__ conn;
  const int32_t* __restrict__ allptr;
  const int32_t* __restrict__ allinc;
  const double* __restrict__ gc;
  const double* __restrict__ lam;   // [N,3]
  double* out;                      // [N,3] (accumulated)
  double mu, kappa, p;
  int64_t ne;
  int32_t n_nodes;
};

// Element quantities at Gauss point g: w, F, F^-1, J, J0^-1, Lam.
template <int NN>
__device__ __forceinline__ void adj_gauss(const AdjParams& P, const int32_t* cn, int g, double& w, double F[9],
                                          double iF[9], double& J, double iJ[9], double Lam[9]) {
  double J0[9], Ju[9], Jl[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) J0[i] = Ju[i] = Jl[i] = 0.0;
#pragma unroll
  for (int b = 0; b < NN; ++b) {
    const int32_t c = cn[b];
    const unsigned mb = P.mask[c];
    const int32_t rb = P.rdof[c];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double x = P.X[3 * (int64_t)c + i], u = node_u(P.gc, rb, mb, i), l = P.lam[3 * (int64_t)c + i];
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const double d = Elem<NN>::dxi(g, b, m);
        J0[3 * i + m] += x * d;
        Ju[3 * i + m] += u * d;
        Jl[3 * i + m] += l * d;
      }
    }
  }
  w = inv3(J0, iJ) * Elem<NN>::wq(g);
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      F[3 * I + i] = (I == i ? 1.0 : 0.0) + Ju[3 * I] * iJ[i] + Ju[3 * I + 1] * iJ[3 + i] + Ju[3 * I + 2] * iJ[6 + i];
      Lam[3 * I + i] = Jl[3 * I] * iJ[i] + Jl[3 * I + 1] * iJ[3 + i] + Jl[3 * I + 2] * iJ[6 + i];
    }
  J = inv3(F, iF);
}

// M of the formula above (row-major M[p][k]) and dPhi/dmu at one Gauss point.
__device__ __forceinline__ void adj_M(const double F[9], const double iF[9], double J, const double Lam[9], double mu,
                                      double kappa, double M[9], double& dmu) {
  const double Jm = jm23(J);
  double sF2 = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
  const double I1 = Jm * sF2, muJm = mu * Jm;
  const double c2 = kappa * J * (J - 1.0) - mu * I1 / 3.0;
  // P[I][i] = s[i][I] = muJm F[I][i] + c2 iF[i][I]
  double Pm[9];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int i = 0; i < 3; ++i) Pm[3 * I + i] = muJm * F[3 * I + i] + c2 * iF[3 * i + I];
  double PL = 0.0, FL = 0.0, tr = 0.0, dmu_g = 0.0;
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      PL += Pm[3 * I + i] * Lam[3 * I + i];
      FL += F[3 * I + i] * Lam[3 * I + i];
      tr += iF[3 * i + I] * Lam[3 * I + i];                      // tr(F^-1 Lam)
      dmu_g += (Jm * F[3 * I + i] - I1 / 3.0 * iF[3 * i + I]) * Lam[3 * I + i];
    }
  dmu = dmu_g;
  // ds[i][j] = T1_ij tr + T2_ij FL + (T3 Lam iF)_ij + muJm Lam[j][i]; A[Lam][I][i] = ds[i][I]
  const double a1 = -2.0 / 3.0 * muJm;                              // T1 = a1 F^T + b1 iF
  const double b1 = kappa * J * (2.0 * J - 1.0) + 2.0 / 9.0 * mu * I1;
  const double t3 = mu * I1 / 3.0 - kappa * J * (J - 1.0);          // T3 = t3 iF, T2 = a1 iF
  double LiF[9];                                                    // Lam iF
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) LiF[3 * k + j] = Lam[3 * k] * iF[j] + Lam[3 * k + 1] * iF[3 + j] + Lam[3 * k + 2] * iF[6 + j];
  double A[9];                                                      // A[Lam][I][i] = ds[i][I]
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double T1 = a1 * F[3 * j + i] + b1 * iF[3 * i + j];
      const double T2 = a1 * iF[3 * i + j];
      const double T3L = t3 * (iF[3 * i] * LiF[j] + iF[3 * i + 1] * LiF[3 + j] + iF[3 * i + 2] * LiF[6 + j]);
      A[3 * j + i] = T1 * tr + T2 * FL + T3L + muJm * Lam[3 * j + i];
    }
  // M = PL I - (F - I)^T A - Lam^T P
#pragma unroll
  for (int pp = 0; pp < 3; ++pp)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double v = (pp == k ? PL : 0.0);
#pragma unroll
      for (int I = 0; I < 3; ++I) v -= (F[3 * I + pp] - (I == pp ? 1.0 : 0.0)) * A[3 * I + k] + Lam[3 * I + pp] * Pm[3 * I + k];
      M[3 * pp + k] = v;
    }
}

// dPhi/dX for every node: one thread per node over all its incidences.
template <int NN>
__global__ void __launch_bounds__(128) k_vjp_vol(AdjParams P) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int q = P.allptr[n]; q < P.allptr[n + 1]; ++q) {
    const int ea = P.allinc[q];
    const int64_t e = ea >> 4;
    const int a = ea & 15;
    int32_t cn[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
#pragma unroll
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double w, F[9], iF[9], J, iJ[9], Lam[9], M[9], dmu;
      adj_gauss<NN>(P, cn, g, w, F, iF, J, iJ, Lam);
      adj_M(F, iF, J, Lam, P.mu, P.kappa, M, dmu);
      double ga[3];
      const double d0 = Elem<NN>::dxi(g, a, 0), d1 = Elem<NN>::dxi(g, a, 1), d2 = Elem<NN>::dxi(g, a, 2);
#pragma unroll
      for (int i = 0; i < 3; ++i) ga[i] = d0 * iJ[i] + d1 * iJ[3 + i] + d2 * iJ[6 + i];
#pragma unroll
      for (int pp = 0; pp < 3; ++pp) acc[pp] += w * (M[3 * pp] * ga[0] + M[3 * pp + 1] * ga[1] + M[3 * pp + 2] * ga[2]);
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) P.out[3 * (int64_t)n + i] += acc[i];
}

// dPhi/dmu: element-parallel, fixed-order two-level sum.
template <int NN>
__global__ void __launch_bounds__(256) k_vjp_mu(AdjParams P, double* partial) {
  __shared__ double sh[256];
  const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (e < P.ne) {
    int32_t cn[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
#pragma unroll
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double w, F[9], iF[9], J, iJ[9], Lam[9], M[9], dmu;
      adj_gauss<NN>(P, cn, g, w, F, iF, J, iJ, Lam);
      adj_M(F, iF, J, Lam, P.mu, P.kappa, M, dmu);
      acc += w * dmu;
    }
  }
  double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_sum_partials_adj(const double* __restrict__ partial, int64_t n, double* out) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 256) acc += partial[i];
  double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) out[0] = s;
}

template <int NF>
struct AFace;
template <>
struct AFace<3> {
  static constexpr int NG = 3;
  __device__ static __forceinline__ double sf(int g, int m, int a) { return c_sf_t3[g][m][a]; }
  __device__ static __forceinline__ double w(int g) { return c_w_t3[g]; }
};
template <>
struct AFace<4> {
  static constexpr int NG = 4;
  __device__ static __forceinline__ double sf(int g, int m, int a) { return c_sf_q4[g][m][a]; }
  __device__ static __forceinline__ double w(int g) { return c_w_q4[g]; }
};

// p d2V/dx2 v for every node of a face group, one thread per node:
// (K_ab v_b)[i] = sum_g p w/3 (A_i (C(b) . v_b) - D_i(b) (B . v_b)), the same
// per-Gauss-point factors as the pressure stiffness kernel.
template <int NF>
__global__ void __launch_bounds__(128) k_face_hvp(AdjParams P, const double* __restrict__ Xi) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int q = P.allptr[n]; q < P.allptr[n + 1]; ++q) {
    const int ea = P.allinc[q];
    const int64_t f = ea >> 4;
    const int a = ea & 15;
    double x[NF][3], v[NF][3];
#pragma unroll
    for (int b = 0; b < NF; ++b) {
      const int32_t c = P.conn[f * NF + b];
      const unsigned mb = P.mask[c];
      const int32_t rb = P.rdof[c];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        x[b][i] = Xi[3 * (int64_t)c + i] + node_u(P.gc, rb, mb, i);
        v[b][i] = P.lam[3 * (int64_t)c + i];
      }
    }
#pragma unroll
    for (int g = 0; g < AFace<NF>::NG; ++g) {
      double r[9], inv[9];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          double s = 0.0;
#pragma unroll
          for (int b = 0; b < NF; ++b) s += AFace<NF>::sf(g, m, b) * x[b][i];
          r[3 * i + m] = s;
        }
      const double det = inv3(r, inv);
      const double w3 = AFace<NF>::w(g) / 3.0 * P.p;
      double A[3], B[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double sa = 0.0, sb = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          sa += AFace<NF>::sf(g, m, a) * det * inv[3 * m + i];
          sb += AFace<NF>::sf(g, m, a) * inv[3 * m + i];
        }
        A[i] = sa;
        B[i] = sb;
      }
#pragma unroll
      for (int b = 0; b < NF; ++b) {
        double C[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double sc = 0.0;
#pragma unroll
          for (int m = 0; m < 3; ++m) sc += AFace<NF>::sf(g, m, b) * inv[3 * m + j];
          C[j] = sc;
        }
        const double Cv = C[0] * v[b][0] + C[1] * v[b][1] + C[2] * v[b][2];
        const double Bv = B[0] * v[b][0] + B[1] * v[b][1] + B[2] * v[b][2];
#pragma unroll
        for (int i = 0; i < 3; ++i) acc[i] += w3 * (A[i] * Cv - det * C[i] * Bv);
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) P.out[3 * (int64_t)n + i] += acc[i];
}

static AdjParams adj_params(const fea_nodes_t* N, const fea_group_t* G, const double* X, const double* gc,
                            const double* lam, double* out) {
  AdjParams P;
  P.X = X;
  P.rdof = N->rdof_dev;
  P.mask = N->mask_dev;
  P.conn = G->conn_dev;
  P.allptr = G->allptr_dev;
  P.allinc = G->allinc_dev;
  P.gc = gc;
  P.lam = lam;
  P.out = out;
  P.mu = P.kappa = P.p = 0.0;
  P.ne = G->ne;
  P.n_nodes = (int32_t)N->n_nodes;
  return P;
}

}  // namespace fea

using namespace fea;

extern "C" int fea_adjoint_vjp_volume(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                      const double* gc, const double* lam, double* dX, double* dmu,
                                      double* scratch, int64_t scratch_len, cudaStream_t st) {
  if (!N || !G || !gc || !lam || !dX || !dmu || !scratch) return FEA_EINVAL;
  if ((G->kind != FEA_C3D4 && G->kind != FEA_C3D8) || !G->allptr_dev || !G->allinc_dev) return FEA_EINVAL;
  if (scratch_len < (G->ne + 255) / 256 + 1) return FEA_EWORK;
  if (int r = ensure_tables()) return r;
  AdjParams P = adj_params(N, G, N->X_dev, gc, lam, dX);
  P.mu = mu;
  P.kappa = kappa;
  const bool hex = G->kind == FEA_C3D8;
  if (N->n_nodes > 0) {
    const int grid = grid_for(N->n_nodes, 128);
    if (hex) k_vjp_vol<8><<<grid, 128, 0, st>>>(P);
    else k_vjp_vol<4><<<grid, 128, 0, st>>>(P);
    count_launch();
  }
  const int64_t nb = (G->ne + 255) / 256;
  if (nb > 0) {
    if (hex) k_vjp_mu<8><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    else k_vjp_mu<4><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    count_launch();
  }
  k_sum_partials_adj<<<1, 256, 0, st>>>(scratch, nb, dmu);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_adjoint_hvp_pressure(const fea_nodes_t* N, const fea_group_t* G, double p, const double* Xi,
                                        const double* gc, const double* v, double* out, cudaStream_t st) {
  if (!N || !G || !Xi || !gc || !v || !out) return FEA_EINVAL;
  if ((G->kind != FEA_T3 && G->kind != FEA_Q4) || !G->allptr_dev || !G->allinc_dev) return FEA_EINVAL;
  if (int r = ensure_tables()) return r;
  if (N->n_nodes == 0) return FEA_OK;
  AdjParams P = adj_params(N, G, Xi, gc, v, out);
  P.p = p;
  const int grid = grid_for(N->n_nodes, 128);
  if (G->kind == FEA_T3) k_face_hvp<3><<<grid, 128, 0, st>>>(P, Xi);
  else k_face_hvp<4><<<grid, 128, 0, st>>>(P, Xi);
  count_launch();
  return (int)cudaGetLastError();
}
