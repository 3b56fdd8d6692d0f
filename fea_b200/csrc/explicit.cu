// Explicit central difference with lumped mass, one fused kernel per step
// (sm_100a).
//
// Replaces the time loop of DynamicExplicitSolver.solve (FEA =
// sssnnn7119/FEA, FEA/solver/dynamic_explicit.py:97-140):
//     vh_{k+1/2} = vh_{k-1/2} + dt a_k
//     u_{k+1}    = u_k + dt vh_{k+1/2}
//     a_{k+1}    = minv * (-f_int(u_{k+1}))          (assemble_force, R0 = -R)
//     v_{k+1}    = (vh_{k+1/2} + vh_{k-1/2}) / 2
// One thread per node evaluates the internal force of the node from its
// incident elements (gather, no atomics) and immediately advances that node's
// state; u is double-buffered so every thread reads a consistent u_k.  The
// element nodes' coordinates and displacements are read from a node-major
// copy (x, y, z, ux, uy, uz per node: three 16-byte loads instead of eight
// scalar loads through the mask and the reduced DOF numbering), double-
// buffered with u and written by each node's thread as it advances.  The
// element math runs in T (double, or float for the FP32 variant) and the
// nodal sums in double.
#include <cmath>

#include "common.cuh"

namespace fea {

struct ExParams {
  const double* __restrict__ X;
  const int32_t* __restrict__ rdof;
  const uint8_t* __restrict__ mask;
  const int32_t* __restrict__ conn;
  const int32_t* __restrict__ inc;
  const int32_t* __restrict__ nodeinc;
  const double* __restrict__ minv;
  const double* __restrict__ u;   // u_k (read by all threads)
  double* unext;                  // u_{k+1}
  double* vh;                     // in: vh_{k-1/2} (or v0 when init), out: vh_{k+1/2}
  double* v;                      // out: v_{k+1}
  double* a;                      // in/out
  const double* __restrict__ xu;  // [N, 6] coordinates and u_k of every node
  double* xunext;                 // [N, 6] the same at u_{k+1}
  double mu, kappa, dt;
  int32_t n_nodes;
};

// residual contribution of local node a of one element, computed in T
template <int NN, class T>
__device__ __forceinline__ void elem_force(const ExParams& P, const int32_t* cn, int a, double r[3]) {
  const T mu = (T)P.mu, kappa = (T)P.kappa;
#pragma unroll
  for (int g = 0; g < Elem<NN>::NG; ++g) {
    T J0[9], Ju[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) J0[i] = Ju[i] = T(0);
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      const double2* xb = reinterpret_cast<const double2*>(P.xu + 6 * (int64_t)cn[b]);
      const double2 v0 = xb[0], v1 = xb[1], v2 = xb[2];
      const T x[3] = {(T)v0.x, (T)v0.y, (T)v1.x}, uu[3] = {(T)v1.y, (T)v2.x, (T)v2.y};
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        T d = (T)Elem<NN>::dxi(g, b, m);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          J0[3 * i + m] += x[i] * d;
          Ju[3 * i + m] += uu[i] * d;
        }
      }
    }
    T iJ[9], F[9], iF[9];
    T det0 = inv3(J0, iJ);
    T w = det0 * (T)Elem<NN>::wq(g);
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        F[3 * I + i] = (I == i ? T(1) : T(0)) + Ju[3 * I] * iJ[i] + Ju[3 * I + 1] * iJ[3 + i] + Ju[3 * I + 2] * iJ[6 + i];
    T J, Jm;
    if constexpr (sizeof(T) == 8 && NN == 4) {       // (C3D8: 222 instead of 168 registers)
      double jmd;
      J = inv3_jm(F, iF, &jmd);
      Jm = jmd;
    } else {
      J = inv3(F, iF);
      Jm = (T)jm23((double)J);
    }
    T sF2 = T(0);
#pragma unroll
    for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
    T I1 = Jm * sF2;
    T muJm = mu * Jm;
    T c2 = kappa * J * (J - T(1)) - mu * I1 / T(3);
    // g_a = iJ^T dxi_a ; f_a = F g_a ; q_a = F^-T g_a
    T ga[3];
    const T d0 = (T)Elem<NN>::dxi(g, a, 0), d1 = (T)Elem<NN>::dxi(g, a, 1), d2 = (T)Elem<NN>::dxi(g, a, 2);
#pragma unroll
    for (int i = 0; i < 3; ++i) ga[i] = d0 * iJ[i] + d1 * iJ[3 + i] + d2 * iJ[6 + i];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T fa = F[3 * j] * ga[0] + F[3 * j + 1] * ga[1] + F[3 * j + 2] * ga[2];
      T qa = iF[j] * ga[0] + iF[3 + j] * ga[1] + iF[6 + j] * ga[2];
      r[j] += (double)(w * (muJm * fa + c2 * qa));
    }
  }
}

// flags: bit0 compute the force (else use a), bit1 init (vh = v0 - dt/2 a),
//        bit2 advance (vh, v, u_next)
template <int NN, class T>
__global__ void __launch_bounds__(128, NN == 4 ? 5 : 1) k_explicit(ExParams P, int flags) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  const unsigned mn = P.mask[n];
  if (!mn) return;
  double r[3] = {0.0, 0.0, 0.0};
  if ((flags & 1) && NN == 8) {
    for (int q = P.nodeinc[n]; q < P.nodeinc[n + 1]; ++q) {
      const int ea = P.inc[q];
      const int64_t e = ea >> 4;
      int32_t cn[NN];
#pragma unroll
      for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
      elem_force<NN, T>(P, cn, ea & 15, r);
    }
  } else if (flags & 1) {
    // C3D4: the next incidence and its element's nodes are loaded while the
    // current element is evaluated (for C3D8 the extra registers cost a CTA
    // per SM)
    const int q0 = P.nodeinc[n], q1 = P.nodeinc[n + 1];
    int ea_n = 0;
    int32_t cn_n[NN];
    if (q0 < q1) {
      ea_n = P.inc[q0];
#pragma unroll
      for (int b = 0; b < NN; ++b) cn_n[b] = P.conn[(int64_t)(ea_n >> 4) * NN + b];
    }
    for (int q = q0; q < q1; ++q) {
      const int ea = ea_n;
      int32_t cn[NN];
#pragma unroll
      for (int b = 0; b < NN; ++b) cn[b] = cn_n[b];
      if (q + 1 < q1) {
        ea_n = P.inc[q + 1];
#pragma unroll
        for (int b = 0; b < NN; ++b) cn_n[b] = P.conn[(int64_t)(ea_n >> 4) * NN + b];
      }
      elem_force<NN, T>(P, cn, ea & 15, r);
    }
  }
  const int32_t base = P.rdof[n];
  int rj = 0;
  double un[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (!(mn >> d & 1u)) continue;
    const int32_t i = base + rj++;
    double acc = (flags & 1) ? -P.minv[i] * r[d] : P.a[i];
    if (flags & 1) P.a[i] = acc;
    if (flags & 4) {
      double vh = (flags & 2) ? P.vh[i] - 0.5 * P.dt * acc : P.vh[i];
      double vhn = vh + P.dt * acc;
      P.v[i] = 0.5 * (vhn + vh);
      P.vh[i] = vhn;
      un[d] = P.u[i] + P.dt * vhn;
      P.unext[i] = un[d];
    } else if (flags & 2) {
      P.vh[i] = P.vh[i] - 0.5 * P.dt * acc;
    }
  }
  if (flags & 4) {                               // the node's copy at u_{k+1} (fixed components 0)
    double* o = P.xunext + 6 * (int64_t)n;
    o[3] = un[0];
    reinterpret_cast<double2*>(o)[2] = make_double2(un[1], un[2]);
  }
}

// The node-major copy of coordinates and u (both buffers): x, y, z, then
// the displacement (0 for fixed components).
__global__ void __launch_bounds__(256) k_xu_init(ExParams P, double* __restrict__ xu0, double* __restrict__ xu1) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  const unsigned m = P.mask[n];
  const int32_t rd = P.rdof[n];
  const double* x = P.X + 3 * (int64_t)n;
  const double2 a = make_double2(x[0], x[1]), b = make_double2(x[2], node_u(P.u, rd, m, 0)),
                c = make_double2(node_u(P.u, rd, m, 1), node_u(P.u, rd, m, 2));
  double2* o0 = reinterpret_cast<double2*>(xu0 + 6 * (int64_t)n);
  double2* o1 = reinterpret_cast<double2*>(xu1 + 6 * (int64_t)n);
  o0[0] = a; o0[1] = b; o0[2] = c;
  o1[0] = a; o1[1] = b; o1[2] = c;
}

// One stage of the central-difference loop around a separately assembled
// residual (several element groups, loads): see fea_explicit_stage.
__global__ void __launch_bounds__(256) k_explicit_stage(int64_t n, int32_t stage, double dt,
                                                        const double* __restrict__ minv,
                                                        const double* __restrict__ R, double* __restrict__ u,
                                                        double* __restrict__ vh, double* __restrict__ vhp,
                                                        double* __restrict__ a, double* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (stage == 0) {                       // before the force pass
      const double h = vh[i];
      const double hn = h + dt * a[i];
      vhp[i] = h;
      vh[i] = hn;
      u[i] = u[i] + dt * hn;
    } else if (stage == 1) {                // after it
      a[i] = -minv[i] * R[i];
      v[i] = 0.5 * (vh[i] + vhp[i]);
    } else {                                // start: a_0 and vh_{-1/2}
      const double ai = -minv[i] * R[i];
      a[i] = ai;
      vh[i] = v[i] - 0.5 * dt * ai;
    }
  }
}

}  // namespace fea

using namespace fea;

extern "C" int fea_explicit_stage(int64_t n, int32_t stage, double dt, const double* minv, const double* R,
                                  double* u, double* vh, double* vhp, double* a, double* v, cudaStream_t st) {
  if (n < 0 || stage < 0 || stage > 2 || !minv || !vh || !a) return FEA_EINVAL;
  if (stage == 0 && (!u || !vhp)) return FEA_EINVAL;
  if (stage >= 1 && !R) return FEA_EINVAL;
  if ((stage == 1 && (!vhp || !v)) || (stage == 2 && !v)) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n + 255) / 256;
  const int grid = (int)(want < 8LL * sms ? want : 8LL * sms);
  k_explicit_stage<<<grid, 256, 0, st>>>(n, stage, dt, minv, R, u, vh, vhp, a, v);
  count_launch();
  return (int)cudaGetLastError();
}

// second u buffer (ndof doubles, rounded to 16 bytes), then the two
// node-major copies of coordinates and u (6 doubles per node each)
extern "C" int64_t fea_explicit_work_len(const fea_nodes_t* N) {
  if (!N || N->ndof < 0 || N->n_nodes < 0) return 0;
  return ((N->ndof + 1) & ~(int64_t)1) + 12 * N->n_nodes;
}

// state on entry: u = u_k, vh = vh_{k-1/2}, a = a_k   (init == 0), or
//                 u = u_0, v = v_0 (a, vh are outputs)  (init != 0)
extern "C" int fea_explicit_run(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                   const double* minv, double dt, int64_t steps, int32_t fp32, int32_t init,
                                   double* u, double* vh, double* a, double* v, double* work, int64_t work_len,
                                   cudaStream_t st) {
  if (!N || !G || !minv || !u || !vh || !a || !v || !work || steps < 0) return FEA_EINVAL;
  if (G->kind != FEA_C3D4 && G->kind != FEA_C3D8) return FEA_EINVAL;
  if (work_len < fea_explicit_work_len(N)) return FEA_EWORK;
  if (((uintptr_t)work & 15) != 0) return FEA_EINVAL;
  if (int r = ensure_tables()) return r;
  if (N->n_nodes == 0 || N->ndof == 0) return FEA_OK;
  ExParams P;
  P.X = N->X_dev;
  P.rdof = N->rdof_dev;
  P.mask = N->mask_dev;
  P.conn = G->conn_dev;
  P.inc = G->inc_dev;
  P.nodeinc = G->nodeinc_dev;
  P.minv = minv;
  P.vh = vh;
  P.v = v;
  P.a = a;
  P.mu = mu;
  P.kappa = kappa;
  P.dt = dt;
  P.n_nodes = (int32_t)N->n_nodes;
  double* xub[2] = {work + ((N->ndof + 1) & ~(int64_t)1), work + ((N->ndof + 1) & ~(int64_t)1) + 6 * N->n_nodes};
  P.u = u;
  k_xu_init<<<grid_for(N->n_nodes, 256), 256, 0, st>>>(P, xub[0], xub[1]);
  count_launch();
  const int grid = grid_for(N->n_nodes, 128);
  const bool hex = G->kind == FEA_C3D8;
  auto launch = [&](const double* ucur, double* unext, int flags) {
    P.u = ucur;
    P.unext = unext;
    P.xu = xub[ucur == u ? 0 : 1];
    P.xunext = xub[ucur == u ? 1 : 0];
    if (hex) {
      if (fp32) k_explicit<8, float><<<grid, 128, 0, st>>>(P, flags);
      else k_explicit<8, double><<<grid, 128, 0, st>>>(P, flags);
    } else {
      if (fp32) k_explicit<4, float><<<grid, 128, 0, st>>>(P, flags);
      else k_explicit<4, double><<<grid, 128, 0, st>>>(P, flags);
    }
    count_launch();
  };
  double* buf[2] = {u, work};
  int cur = 0;
  if (init) {
    // v = v0 on entry; v is overwritten with v_1 only when advancing
    if (steps == 0) {
      // a_0 = minv (-f(u_0)); vh_{-1/2} = v0 - dt/2 a_0 ; v stays v0
      cudaMemcpyAsync(vh, v, sizeof(double) * N->ndof, cudaMemcpyDeviceToDevice, st);
      launch(u, work, 1 | 2);
      return (int)cudaGetLastError();
    }
    cudaMemcpyAsync(vh, v, sizeof(double) * N->ndof, cudaMemcpyDeviceToDevice, st);
    launch(buf[cur], buf[1 - cur], 1 | 2 | 4);
  } else {
    if (steps == 0) return FEA_OK;
    launch(buf[cur], buf[1 - cur], 4);   // advance with the given a_k
  }
  cur = 1 - cur;
  for (int64_t k = 1; k < steps; ++k) {
    launch(buf[cur], buf[1 - cur], 1 | 4);
    cur = 1 - cur;
  }
  launch(buf[cur], nullptr, 1);            // a at the final state
  if (cur == 1) cudaMemcpyAsync(u, work, sizeof(double) * N->ndof, cudaMemcpyDeviceToDevice, st);
  return (int)cudaGetLastError();
}

