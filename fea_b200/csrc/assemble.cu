// Element residual / tangent assembly, follower pressure, energy and lumped
// mass for C3D4 / C3D8 Neo-Hookean groups (sm_100a, FP64).
//
// Assembly is a per-node-row GATHER: every (row node n, incident element e)
// pair ("incidence") gets one thread, which evaluates the element at all its
// Gauss points and accumulates the 3 x (3 nn) strip K_e[a(n), :] in
// registers.  The strips of one node are summed in shared memory in a fixed
// order (incidence rank), and the chunk's rows — a contiguous range of the
// reduced CSR values — are written to HBM exactly once.  No atomics, no
// colouring, bitwise-deterministic results.
//
// Reference behaviour reproduced (FEA = sssnnn7119/FEA):
//   F, J, J^-2/3, I1          Element_3D.components_Solid   C3base.py:454-480
//   s = P^T, C_ijkl           NeoHookean.material_Constitutive_C3
//                                                   materials/hyperelastic.py:35-84
//   R_e, K_e, slot scatter    Element_3D.structural_Force   C3base.py:413-452
//   reduced R, K              Assembly._assemble_*_Matrix   assembly.py:311-387
// The kernel never forms the 81-entry C: with alpha = -2/3 mu J^-2/3,
// beta = kappa J (2J-1) + 2/9 mu I1, gamma = mu I1/3 - kappa J (J-1),
// f_b = F g_b and q_b = F^-T g_b (g_b = dN_b/dX), the reference's
// contraction sum_il C_ijkl g_ai g_bl equals
//   (alpha f_a + beta q_a)_j q_bk + alpha q_aj f_bk + gamma q_ak q_bj
//   + mu J^-2/3 (g_a . g_b) delta_jk.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>

#include "common.cuh"

namespace fea {

struct VolParams {
  const double* __restrict__ X;
  const int32_t* __restrict__ rdof;
  const uint8_t* __restrict__ mask;
  const int64_t* __restrict__ vbase;
  const int32_t* __restrict__ rowlen;
  const int32_t* __restrict__ dbase;
  const int32_t* __restrict__ conn;
  const int32_t* __restrict__ inc;
  const uint16_t* __restrict__ boff;
  const int32_t* __restrict__ nodeinc;
  const int32_t* __restrict__ chunkptr;
  const int32_t* __restrict__ chunkinc;
  const int32_t* __restrict__ chunklist;
  const int32_t* __restrict__ chunkdim;
  const int32_t* __restrict__ soff;
  const int32_t* __restrict__ roff;
  const int64_t* __restrict__ adjptr;
  const int32_t* __restrict__ adjcol;
  const int32_t* __restrict__ adjoff;
  const int64_t* __restrict__ uptr;
  const fea_ublk_t* __restrict__ ublk;
  const int32_t* __restrict__ incpos;
  const int32_t* __restrict__ stagepos;
  const int64_t* __restrict__ region;
  const int32_t* __restrict__ moff;
  const double* __restrict__ gc;
  double* K;
  double* R;
  double* elemR;
  double mu, kappa;
  int64_t ne;
  int32_t maxval;
  int32_t n_nodes;
};

// Kinematics of one element at one Gauss point: w, F, F^-1, J and the two
// gradient maps Mq = J0^-1 F^-1, Mf = J0^-1 F^T (so that q_b = Mq^T dxi_b,
// f_b = Mf^T dxi_b) plus iJ = J0^-1 (g_b = iJ^T dxi_b).
template <int NN>
__device__ __forceinline__ void gauss_kin(const VolParams& P, const int32_t* cn, const unsigned* mk,
                                          const int32_t* rd, int g, double& w, double F[9], double iF[9],
                                          double& J, double iJ[9]) {
  double J0[9], Ju[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) J0[i] = Ju[i] = 0.0;
#pragma unroll
  for (int b = 0; b < NN; ++b) {
    const double* xb = P.X + 3 * (int64_t)cn[b];
    double x0 = __ldg(xb), x1 = __ldg(xb + 1), x2 = __ldg(xb + 2);
    double u0 = node_u(P.gc, rd[b], mk[b], 0), u1 = node_u(P.gc, rd[b], mk[b], 1),
           u2 = node_u(P.gc, rd[b], mk[b], 2);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double d = Elem<NN>::dxi(g, b, m);
      J0[m] += x0 * d; J0[3 + m] += x1 * d; J0[6 + m] += x2 * d;
      Ju[m] += u0 * d; Ju[3 + m] += u1 * d; Ju[6 + m] += u2 * d;
    }
  }
  double det0 = inv3(J0, iJ);
  w = det0 * Elem<NN>::wq(g);
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int i = 0; i < 3; ++i)
      F[3 * I + i] = fma(Ju[3 * I], iJ[i], fma(Ju[3 * I + 1], iJ[3 + i], fma(Ju[3 * I + 2], iJ[6 + i], I == i ? 1.0 : 0.0)));
  J = inv3(F, iF);
}

// Residual strip (3) and, if WK, tangent strip (NN x 9) of local node a.
template <int NN, bool WK>
__device__ __forceinline__ void element_strip(const VolParams& P, const int32_t* cn, int a,
                                              double (*acc)[9], double racc[3]) {
  unsigned mk[NN];
  int32_t rd[NN];
#pragma unroll
  for (int b = 0; b < NN; ++b) {
    mk[b] = P.mask[cn[b]];
    rd[b] = P.rdof[cn[b]];
  }
  racc[0] = racc[1] = racc[2] = 0.0;
  if (WK) {
#pragma unroll
    for (int b = 0; b < NN; ++b)
#pragma unroll
      for (int i = 0; i < 9; ++i) acc[b][i] = 0.0;
  }
  const double mu = P.mu, kappa = P.kappa;
#pragma unroll
  for (int g = 0; g < Elem<NN>::NG; ++g) {
    double w, F[9], iF[9], J, iJ[9];
    gauss_kin<NN>(P, cn, mk, rd, g, w, F, iF, J, iJ);
    double Jm = jm23(J);
    double sF2 = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
    double I1 = Jm * sF2;
    double muJm = mu * Jm;
    double c2 = kappa * J * (J - 1.0) - mu * I1 / 3.0;
    // Mq[m][k] = sum_i iJ[m][i] iF[i][k];  Mf[m][k] = sum_i iJ[m][i] F[k][i]
    double Mq[9], Mf[9];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        Mq[3 * m + k] = iJ[3 * m] * iF[k] + iJ[3 * m + 1] * iF[3 + k] + iJ[3 * m + 2] * iF[6 + k];
        Mf[3 * m + k] = iJ[3 * m] * F[3 * k] + iJ[3 * m + 1] * F[3 * k + 1] + iJ[3 * m + 2] * F[3 * k + 2];
      }
    double da0 = Elem<NN>::dxi(g, a, 0), da1 = Elem<NN>::dxi(g, a, 1), da2 = Elem<NN>::dxi(g, a, 2);
    double qa[3], fa[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      qa[k] = da0 * Mq[k] + da1 * Mq[3 + k] + da2 * Mq[6 + k];
      fa[k] = da0 * Mf[k] + da1 * Mf[3 + k] + da2 * Mf[6 + k];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) racc[j] += w * (muJm * fa[j] + c2 * qa[j]);
    if (WK) {
      double alpha = -2.0 / 3.0 * muJm;
      double beta = kappa * J * (2.0 * J - 1.0) + 2.0 / 9.0 * mu * I1;
      double gamma = mu * I1 / 3.0 - kappa * J * (J - 1.0);
      double va[3], ua[3], ga[3], gm[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        va[j] = w * (alpha * fa[j] + beta * qa[j]);
        ua[j] = w * alpha * qa[j];
        ga[j] = w * gamma * qa[j];
      }
      // g_a = iJ^T dxi_a ; gm = iJ g_a (so that g_a . g_b = gm . dxi_b)
      double gav[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) gav[i] = da0 * iJ[i] + da1 * iJ[3 + i] + da2 * iJ[6 + i];
      double wc = w * muJm;
#pragma unroll
      for (int m = 0; m < 3; ++m) gm[m] = wc * (iJ[3 * m] * gav[0] + iJ[3 * m + 1] * gav[1] + iJ[3 * m + 2] * gav[2]);
      // fused multiply-add chains; the delta term only on the diagonal
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          double h[3];
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            double t = ga[k] * Mq[3 * m + j];
            t = fma(ua[j], Mf[3 * m + k], t);
            t = fma(va[j], Mq[3 * m + k], t);
            h[m] = j == k ? t + gm[m] : t;
          }
#pragma unroll
          for (int b = 0; b < NN; ++b) {
            double t = acc[b][3 * j + k];
            t = fma(Elem<NN>::dxi(g, b, 0), h[0], t);
            t = fma(Elem<NN>::dxi(g, b, 1), h[1], t);
            t = fma(Elem<NN>::dxi(g, b, 2), h[2], t);
            acc[b][3 * j + k] = t;
          }
        }
    }
  }
}

// out[i] (+)= src[i] for i = threadIdx.x, + blockDim.x, ... < len: the global
// reads of eight strides issued together (one round trip per eight values
// instead of one per value: the read-modify-write of the accumulate mode was
// latency-serial)
template <bool ACC>
__device__ __forceinline__ void add_rows(double* __restrict__ out, const double* __restrict__ src, int len) {
  constexpr int U = 8;
  for (int i0 = threadIdx.x; i0 < len; i0 += U * (int)blockDim.x) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      v[u] = (ACC && i < len) ? out[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * (int)blockDim.x;
      if (i < len) out[i] = ACC ? v[u] + src[i] : src[i];
    }
  }
}

// Copy a chunk's shared-memory rows to the reduced K values and R: one flat
// copy when the chunk's node rows are contiguous in HBM, else node by node.
template <bool ACC>
__device__ __forceinline__ void write_back(const int32_t* __restrict__ chunkptr, const int32_t* __restrict__ chunklist,
                                           const int32_t* __restrict__ chunkdim, const int64_t* __restrict__ vbase,
                                           const int32_t* __restrict__ dbase, const uint8_t* __restrict__ mask,
                                           const int32_t* __restrict__ soff, const int32_t* __restrict__ roff, int ch,
                                           const double* sm, double* K, int nv, double* R) {
  const int l0 = chunkptr[ch], l1 = chunkptr[ch + 1];
  const int nr = chunkdim[3 * ch + 1];
  if (chunkdim[3 * ch + 2]) {
    const int n0 = chunklist[l0];
    if (K) {
      add_rows<ACC>(K + vbase[n0], sm, nv);
    }
    if (R) add_rows<ACC>(R + dbase[n0], sm + nv, nr);
    return;
  }
  for (int l = l0; l < l1; ++l) {
    const int n = chunklist[l];
    if (K) {
      add_rows<ACC>(K + vbase[n], sm + soff[n], (int)(vbase[n + 1] - vbase[n]));
    }
    if (R) {
      const int f = popc3(mask[n]);
      if ((int)threadIdx.x < f) {
        double* out = R + dbase[n];
        out[threadIdx.x] = ACC ? out[threadIdx.x] + sm[nv + roff[n] + threadIdx.x] : sm[nv + roff[n] + threadIdx.x];
      }
    }
  }
}

template <int NN>
struct VolTPB { static constexpr int v = NN == 8 ? 128 : 256; };

// R + K gather kernel: one CTA per chunk of consecutive node rows.
template <int NN, bool WR, bool ACC, bool ER>
__global__ void __launch_bounds__(VolTPB<NN>::v) k_vol_rk(VolParams P) {
  extern __shared__ double sm[];
  const int ch = blockIdx.x;
  const int i0 = P.chunkinc[ch], i1 = P.chunkinc[ch + 1];
  const int nv = P.chunkdim[3 * ch];
  const int nr = WR ? P.chunkdim[3 * ch + 1] : 0;
  for (int i = threadIdx.x; i < nv + nr; i += blockDim.x) sm[i] = 0.0;
  __syncthreads();

  const int q = i0 + threadIdx.x;
  const bool act = q < i1;
  double acc[NN][9];
  double racc[3];
  int32_t cn[NN];
  int rank = -1, a = 0, n = 0;
  // the row metadata and column offsets of the incidence, issued before the
  // element math so that their loads overlap it
  unsigned mn = 0, mcb[NN], bob[NN];
  int rowoff = 0, L = 0, dr = 0;
  if (act) {
    const int ea = P.inc[q];
    const int64_t e = ea >> 4;
    a = ea & 15;
#pragma unroll
    for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
    n = cn[a];
    rank = q - P.nodeinc[n];
    mn = P.mask[n];
    rowoff = P.soff[n];
    L = P.rowlen[n];
    dr = P.roff[n];
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      bob[b] = P.boff[(int64_t)q * NN + b];
      mcb[b] = P.mask[cn[b]];
    }
    element_strip<NN, true>(P, cn, a, acc, racc);
    if (ER) {
#pragma unroll
      for (int j = 0; j < 3; ++j) P.elemR[(int64_t)(3 * a + j) * P.ne + e] = racc[j];
    }
  }
  // per-node sums in incidence order (one thread per node per round)
  for (int k = 0; k < P.maxval; ++k) {
    if (rank == k) {
#pragma unroll
      for (int b = 0; b < NN; ++b) {
        const unsigned bo = bob[b];
        if (bo == 0xFFFFu) continue;
        const unsigned mc = mcb[b];
        int rj = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          if (!(mn >> j & 1u)) continue;
          double* row = sm + rowoff + rj * L + bo;
          int rk = 0;
#pragma unroll
          for (int kk = 0; kk < 3; ++kk) {
            if (!(mc >> kk & 1u)) continue;
            row[rk] += acc[b][3 * j + kk];
            ++rk;
          }
          ++rj;
        }
      }
      if (WR) {
        int rj = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
          if (mn >> j & 1u) sm[nv + dr + rj++] += racc[j];
      }
    }
    __syncthreads();
  }
  write_back<ACC>(P.chunkptr, P.chunklist, P.chunkdim, P.vbase, P.dbase, P.mask, P.soff, P.roff, ch, sm, P.K, nv,
                  WR ? P.R : nullptr);
}

// ---- C3D8 R + K: element kernel + staged-block gather -----------------------
// k_hex_elem evaluates every element ONCE: 8 lanes per element, lane g
// computes the kinematics of Gauss point g and the vectors q_b = F^-T g_b,
// f_b = F g_b of all 8 nodes into shared memory; then lane a builds the
// upper-triangular blocks K_ab it owns (circulant assignment: b = a + d mod 8,
// d = 0..3, plus d = 4 for a < 4 — 36 blocks over 8 lanes) with its own row
// vectors in registers,
//   K_ab = sum_g (A_a q_b^T + B_a f_b^T + q_b C_a^T + wc (g_a . g_b) I),
//   A_a = w(alpha f_a + beta q_a), B_a = w alpha q_a, C_a = w gamma q_a,
// and the element residual R_a = sum_g w(mu J^-2/3 f_a + c2 q_a).  Each lane
// then writes its blocks from registers to their staged positions (the
// plan's STAGEPOS), oriented to the upper node block (row node numbered
// lower), and R_a to the incidence's slot of a separate array.  A node's
// staged region lists, block-major, the contributions to each of its upper
// blocks in element order; k_hex_gat copies the region to shared memory with
// coalesced 16-byte copies, sums each upper block's contiguous contributions
// and writes the block into the node's rows and its transpose into the
// column node's rows: every CSR value written once.
// g_b itself is not staged: g_a . g_b = (F^-1 f_a) . (F^T q_b) = f_a . q_b,
// so a (Gauss point, node) slot holds 6 doubles and an element 456: 29,184
// bytes of shared memory per CTA.  Six CTAs per SM: the launch bound holds
// the kernel to 168 registers (64 threads x 6 CTAs x 168 <= 64K), 12 warps
// per SM (k_hex_elem 544.3 -> 474.6 us at 64^3 against 45,568 bytes and five
// CTAs).
constexpr int HX_CTAS = 6;                // resident CTAs per SM the launch bound asks for
constexpr int HX_EPB = 8;                 // elements per CTA
constexpr int HX_TPB = 8 * HX_EPB;        // threads per CTA
constexpr int HX_VB = 6;                  // doubles per (gp, node) vector slot: q, f (16-byte aligned)
constexpr int HX_VG = 50;                 // doubles per Gauss point (8 slots + 2 pad: conflict-free rows)
constexpr int HX_SC = 8 * HX_VG;          // offset of the per-Gauss-point scalars (6 each)
constexpr int HX_EL = HX_SC + 48;         // doubles per element (6 scalars per Gauss point)
constexpr int HX_GW = 4;                  // warps per gather CTA
// Gather lanes per row node: 16 (two nodes per warp: 397.0 against 461.4 us
// with 32 lanes per node at 64^3, where rows hold 27 blocks and regions 36),
// 32 when two regions per warp would not fit the shared memory.
constexpr int HX_LPN = 16;

// Offset of the residual slots in the C3D8 scratch: after the staged blocks,
// rounded to 16 bytes.
__host__ __device__ inline int64_t hx_rslot_base(int64_t nblk) { return (nblk * 9 + 1) & ~(int64_t)1; }
constexpr int HX_GINC = 32;               // chunk capacity of C3D8 plans (the C3D8 kernels read no chunks)

// corner signs of hex node / Gauss point c (brick.py:15-25, 151-160)
__device__ __forceinline__ double csx(int c) { return (((c + 1) >> 1) & 1) ? 1.0 : -1.0; }
__device__ __forceinline__ double csy(int c) { return ((c >> 1) & 1) ? 1.0 : -1.0; }
__device__ __forceinline__ double csz(int c) { return (c >> 2) ? 1.0 : -1.0; }
template <bool ER>
__global__ void __launch_bounds__(HX_TPB, HX_CTAS) k_hex_elem(VolParams P, double* __restrict__ stage,
                                                     double* __restrict__ rslot) {
  __shared__ __align__(16) double sv[HX_EPB * HX_EL];
  const double q3 = 0.57735026918962576451;   // 1/sqrt(3)
  const int le = threadIdx.x >> 3;
  const int lane = threadIdx.x & 7;
  const int64_t e = (int64_t)blockIdx.x * HX_EPB + le;
  const bool act = e < P.ne;
  double* V = sv + le * HX_EL;
  // ---- phase 0: node `lane`'s coordinates and displacement, once per element,
  // to the scalar area of V (48 doubles: 6 per node) for all 8 lanes --------
  int32_t cl = 0;
  if (act) {
    cl = P.conn[e * 8 + lane];
    const double* xb = P.X + 3 * (int64_t)cl;
    const unsigned mb = P.mask[cl];
    const int32_t rb = P.rdof[cl];
    double2* o = reinterpret_cast<double2*>(V + HX_SC + lane * 6);
    o[0] = make_double2(__ldg(xb), __ldg(xb + 1));
    o[1] = make_double2(__ldg(xb + 2), node_u(P.gc, rb, mb, 0));
    o[2] = make_double2(node_u(P.gc, rb, mb, 1), node_u(P.gc, rb, mb, 2));
  }
  __syncwarp();
  // ---- phase 1: Gauss point g = lane ----------------------------------------
  const double px = csx(lane) * q3, py = csy(lane) * q3, pz = csz(lane) * q3;
  const double fxp = 1.0 + px, fxm = 1.0 - px, fyp = 1.0 + py, fym = 1.0 - py, fzp = 1.0 + pz, fzm = 1.0 - pz;
  double J0[9], Ju[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) J0[i] = Ju[i] = 0.0;
  // dN_b/dxi at this Gauss point, once for both node loops: 12 products of
  // two shape factors (with the 1/8), signed per node (the same bits as
  // 0.125 * s * f * f')
  double dxs[8][3];
  {
    const double yz[4] = {0.125 * fym * fzm, 0.125 * fyp * fzm, 0.125 * fym * fzp, 0.125 * fyp * fzp};
    const double xz[4] = {0.125 * fxm * fzm, 0.125 * fxp * fzm, 0.125 * fxm * fzp, 0.125 * fxp * fzp};
    const double xy[4] = {0.125 * fxm * fym, 0.125 * fxp * fym, 0.125 * fxm * fyp, 0.125 * fxp * fyp};
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const int ix = ((b + 1) >> 1) & 1, iy = (b >> 1) & 1, iz = b >> 2;
      dxs[b][0] = ix ? yz[iy + 2 * iz] : -yz[iy + 2 * iz];
      dxs[b][1] = iy ? xz[ix + 2 * iz] : -xz[ix + 2 * iz];
      dxs[b][2] = iz ? xy[ix + 2 * iy] : -xy[ix + 2 * iy];
    }
  }
  if (act) {
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const double d0 = dxs[b][0], d1 = dxs[b][1], d2 = dxs[b][2];
      const double2* xs = reinterpret_cast<const double2*>(V + HX_SC + b * 6);
      const double2 v0 = xs[0], v1 = xs[1], v2 = xs[2];
      const double xv[3] = {v0.x, v0.y, v1.x}, uv[3] = {v1.y, v2.x, v2.y};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double x = xv[i], u = uv[i];
        J0[3 * i] += x * d0; J0[3 * i + 1] += x * d1; J0[3 * i + 2] += x * d2;
        Ju[3 * i] += u * d0; Ju[3 * i + 1] += u * d1; Ju[3 * i + 2] += u * d2;
      }
    }
  }
  __syncwarp();                                  // the node data are read: the area takes the scalars
  if (act) {
    double iJ[9], F[9], iF[9];
    const double w = inv3(J0, iJ);             // Gauss weight 1
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        F[3 * I + i] = fma(Ju[3 * I], iJ[i], fma(Ju[3 * I + 1], iJ[3 + i], fma(Ju[3 * I + 2], iJ[6 + i], I == i ? 1.0 : 0.0)));
    double Jm;
    const double J = inv3_jm(F, iF, &Jm);      // F^-1 and J^-2/3 from one reciprocal cube root
    const double mu = P.mu, kappa = P.kappa;
    double sF2 = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
    const double I1 = Jm * sF2, muJm = mu * Jm;
    double* S = V + HX_SC + lane * 6;
    S[0] = w * (-2.0 / 3.0 * muJm);                                 // w alpha
    S[1] = w * (kappa * J * (2.0 * J - 1.0) + 2.0 / 9.0 * mu * I1);  // w beta
    S[2] = w * (mu * I1 / 3.0 - kappa * J * (J - 1.0));              // w gamma
    S[3] = w * muJm;                                                 // w c (delta term, residual)
    S[4] = w * (kappa * J * (J - 1.0) - mu * I1 / 3.0);              // w c2 (residual)
    S[5] = (double)cl;                                               // node `lane`, for phase 3
    // Mq = J0^-1 F^-1, Mf = J0^-1 F^T: q_b = Mq^T dxi_b, f_b = Mf^T dxi_b, g_b = J0^-T dxi_b
    double Mq[9], Mf[9];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        Mq[3 * m + k] = iJ[3 * m] * iF[k] + iJ[3 * m + 1] * iF[3 + k] + iJ[3 * m + 2] * iF[6 + k];
        Mf[3 * m + k] = iJ[3 * m] * F[3 * k] + iJ[3 * m + 1] * F[3 * k + 1] + iJ[3 * m + 2] * F[3 * k + 2];
      }
    double* Vg = V + lane * HX_VG;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const double d0 = dxs[b][0], d1 = dxs[b][1], d2 = dxs[b][2];
      double v[6];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        v[k] = d0 * Mq[k] + d1 * Mq[3 + k] + d2 * Mq[6 + k];
        v[3 + k] = d0 * Mf[k] + d1 * Mf[3 + k] + d2 * Mf[6 + k];
      }
      double2* o = reinterpret_cast<double2*>(Vg + b * HX_VB);   // 16-byte aligned slot
      o[0] = make_double2(v[0], v[1]);
      o[1] = make_double2(v[2], v[3]);
      o[2] = make_double2(v[4], v[5]);
    }
  }
  __syncwarp();
  // ---- phase 2: row node a = lane (lanes of an inactive element idle) --------
  const int a = lane;
  const int nb = a < 4 ? 5 : 4;
  int32_t spos[5] = {-1, -1, -1, -1, -1};      // staged positions of the lane's blocks, loaded early
  int32_t ipos = -1;
  if (act) {
    const int32_t* sp = P.stagepos + e * 36 + (a < 4 ? 5 * a : 20 + 4 * (a - 4));
#pragma unroll
    for (int d = 0; d < 5; ++d)
      if (d < nb) spos[d] = sp[d];
    ipos = P.incpos[e * 8 + a];
  }
  double acc[5][9];
  double racc[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int d = 0; d < 5; ++d)
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[d][i] = 0.0;
#pragma unroll 1
  for (int g = 0; g < (act ? 8 : 0); ++g) {
    const double2* S2 = reinterpret_cast<const double2*>(V + HX_SC + g * 6);   // 16-byte aligned
    const double2 s01 = S2[0], s23 = S2[1], s45 = S2[2];
    const double wa = s01.x, wb = s01.y, wg = s23.x, wc = s23.y, wc2 = s45.x;
    const double* Va = V + g * HX_VG + a * HX_VB;
    double qa[3], fa[3], gm[3], A[3], B[3], Cc[3];
    {
      const double2* v2 = reinterpret_cast<const double2*>(Va);
      const double2 x0 = v2[0], x1 = v2[1], x2 = v2[2];
      qa[0] = x0.x; qa[1] = x0.y; qa[2] = x1.x; fa[0] = x1.y; fa[1] = x2.x; fa[2] = x2.y;
      gm[0] = wc * fa[0]; gm[1] = wc * fa[1]; gm[2] = wc * fa[2];       // w mu J^-2/3 f_a
    }
    double AC[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      A[k] = wa * fa[k] + wb * qa[k];
      B[k] = wa * qa[k];
      Cc[k] = wg * qa[k];
      AC[k] = A[k] + Cc[k];
      racc[k] = fma(wc, fa[k], racc[k]);
      racc[k] = fma(wc2, qa[k], racc[k]);
    }
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      const double* Vb = V + g * HX_VG + ((a + d) & 7) * HX_VB;
      double qb[3], fb[3];
      {
        const double2* v2 = reinterpret_cast<const double2*>(Vb);
        const double2 x0 = v2[0], x1 = v2[1], x2 = v2[2];
        qb[0] = x0.x; qb[1] = x0.y; qb[2] = x1.x; fb[0] = x1.y; fb[1] = x2.x; fb[2] = x2.y;
      }
      const double dg = gm[0] * qb[0] + gm[1] * qb[1] + gm[2] * qb[2];    // w mu J^-2/3 g_a . g_b
      // three fused multiply-adds into each accumulator, the delta term on
      // the diagonal alone: 33 FP64 operations per block and Gauss point.
      // d = 0 (K_aa = wa (f q^T + q f^T) + (wb + wg) q q^T + dg I, symmetric)
      // takes the upper triangle with two FMAs an entry (18), d = 4 the upper
      // triangle (24): at d = 4 every lane computes one, lane a < 4 that of K_a,a+4 and
      // lane a + 4 that of K_a+4,a, whose strict part is the strict lower
      // triangle of K_a,a+4 transposed (the two lanes share the block)
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if ((d == 0 || d == 4) && k < j) continue;
          double t = acc[d][3 * j + k];
          if (d == 0) {                          // K_aa: fa_j B_k + qa_j (A_k + C_k), two FMAs
            t = fma(fa[j], B[k], t);
            t = fma(qa[j], AC[k], t);
          } else {
            t = fma(A[j], qb[k], t);
            t = fma(B[j], fb[k], t);
            t = fma(qb[j], Cc[k], t);
          }
          acc[d][3 * j + k] = t;
        }
      acc[d][0] += dg;
      acc[d][4] += dg;
      acc[d][8] += dg;
    }
  }
  // the strict lower triangle of K_a,a+4 from lane a + 4 (all lanes shuffle)
  const int partner = (lane + 4) & 7;
  const double l10 = __shfl_sync(0xffffffffu, acc[4][1], partner, 8);
  const double l20 = __shfl_sync(0xffffffffu, acc[4][2], partner, 8);
  const double l21 = __shfl_sync(0xffffffffu, acc[4][5], partner, 8);
  acc[0][3] = acc[0][1];
  acc[0][6] = acc[0][2];
  acc[0][7] = acc[0][5];
  acc[4][3] = l10;
  acc[4][6] = l20;
  acc[4][7] = l21;
  // ---- phase 3: every block from registers to its staged position ------------
  // K_ab as computed when the column node is numbered above the row node (or
  // b = a), transposed when below, K_ab + K_ab^T when the element repeats
  // the node (a != b); R_a to the incidence's residual slot.
  if (act) {
    const double na = V[HX_SC + a * 6 + 5];
#pragma unroll
    for (int d = 0; d < 5; ++d) {
      if (d == 4 && nb == 4) break;
      if (spos[d] < 0) continue;
      const double nc = V[HX_SC + ((a + d) & 7) * 6 + 5];
      double* out = stage + (int64_t)spos[d] * 9;
      if (d == 0 || nc > na) {
#pragma unroll
        for (int i = 0; i < 9; ++i) out[i] = acc[d][i];
      } else if (nc < na) {
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int k = 0; k < 3; ++k) out[3 * j + k] = acc[d][3 * k + j];
      } else {
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int k = 0; k < 3; ++k) out[3 * j + k] = acc[d][3 * j + k] + acc[d][3 * k + j];
      }
    }
    if (ipos >= 0) {
      double2* ro = reinterpret_cast<double2*>(rslot + (int64_t)ipos * 4);
      ro[0] = make_double2(racc[0], racc[1]);
      ro[1] = make_double2(racc[2], 0.0);
    }
  }
  if (ER && act) {
#pragma unroll
    for (int j = 0; j < 3; ++j) P.elemR[(int64_t)(3 * a + j) * P.ne + e] = racc[j];
  }
}

// Per node row: a group of LPN lanes per row node n.  The group copies the
// node's region (its staged contributions, block-major) and its residual
// slots to shared memory with 16-byte asynchronous copies; then one lane per
// upper node block (n, c >= n), from the block's record, sums its
// contributions (element order, fixed), writes the 3x3 (free DOFs only)
// into the node's contiguous CSR rows and, for c != n, the transpose into
// c's rows; the diagonal lane writes the node's residual, the sum of its
// slots in incidence (element) order.  The records are loaded while the
// copies are in flight.  FIXED (regular meshes): region, records and slots
// sit at n * capb, 16 n and n * capq, so the copies and record loads do not
// wait for the node's metadata.  capb = the largest region, capq = the most
// incidences of a node (shared memory per group: capb blocks and capq
// slots).
template <bool WR, bool ACC, int LPN, bool FIXED>
__global__ void __launch_bounds__(HX_GW * 32, 8) k_hex_gat(VolParams P, const double* __restrict__ stage,
                                                        const double* __restrict__ rslot, int capb, int capq) {
  extern __shared__ __align__(16) double gsm[];
  static_assert(LPN == 8 || LPN == 16 || LPN == 32, "lanes per node");
  constexpr int NPW = 32 / LPN;                   // nodes per warp
  const int warp = threadIdx.x >> 5;
  const int sub = (threadIdx.x & 31) / LPN;
  const int lane = (threadIdx.x & 31) % LPN;      // lane within the node's group
  const unsigned gmask = LPN == 32 ? 0xffffffffu : (((1u << LPN) - 1u) << (sub * LPN));
  const int64_t n = ((int64_t)blockIdx.x * HX_GW + warp) * NPW + sub;
  if (n >= P.n_nodes) return;
  // the node's metadata issued together, before the mask decides; in the
  // fixed layout the region, record and residual-slot addresses follow from
  // n alone, so their copies start without waiting for these loads
  const unsigned mn = P.mask[n];
  const int64_t b0 = FIXED ? n * capb : P.region[n], b1 = FIXED ? b0 + capb : P.region[n + 1];
  const int64_t u0 = FIXED ? n * 16 : P.uptr[n], u1 = FIXED ? u0 + 16 : P.uptr[n + 1];
  const int q0 = P.nodeinc[n], q1 = P.nodeinc[n + 1];
  const int L = P.rowlen[n];                     // before the copy: no load waits behind its barrier
  const int32_t rdn = P.rdof[n];
  if (!FIXED && !mn) return;
  const int nbk = b1 - b0 < capb ? (int)(b1 - b0) : capb;
  const int64_t nu = u1 - u0;
  const int64_t rs0 = FIXED ? n * capq : q0;     // the node's first residual slot
  const int nqc = FIXED ? capq : (q1 - q0 < capq ? q1 - q0 : capq);   // slots copied
  // the lane's first record: targets (row, transpose) and (rowlen_c, mask_c, first, count)
  int64_t u = lane;
  longlong2 tg = make_longlong2(0, 0);
  int4 mt = make_int4(0, 0, 0, 0);
  if (u < nu) {
    const longlong2* r = reinterpret_cast<const longlong2*>(P.ublk + u0 + u);
    tg = r[0];
    mt = *reinterpret_cast<const int4*>(r + 1);
  }
  // the group's shared area: the region (capb blocks), then the node's
  // residual slots (capq x 4 doubles) when R is written
  double* S = gsm + (int64_t)(warp * NPW + sub) * (capb * 9 + (WR ? capq * 4 : 0));
  double* SR = S + capb * 9;
  {
    // regions start at even blocks and hold an even number, residual slots
    // are 32 bytes: whole 16-byte pieces, copied through L2 only (cg)
    const double* src = stage + b0 * 9;
    const int nd2 = (nbk * 9) >> 1;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(S);
    for (int i = lane; i < nd2; i += LPN)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sbase + 16u * (unsigned)i), "l"(src + 2 * i)
                   : "memory");
    if (WR) {
      const double* rsrc = rslot + rs0 * 4;
      const unsigned rbase = (unsigned)__cvta_generic_to_shared(SR);
      for (int i = lane; i < 2 * nqc; i += LPN)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(rbase + 16u * (unsigned)i),
                     "l"(rsrc + 2 * i)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  }
  __syncwarp(gmask);
  if (FIXED && !mn) return;                      // (the whole group: mn is the group's node's)
  const int nq = q1 - q0 < capq ? q1 - q0 : capq;
  while (u < nu) {
    if (FIXED && tg.x < 0) break;                // the node's records are first in its 16 slots
    double blk[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) blk[i] = 0.0;
    const int k1 = min(mt.z + mt.w, nbk);        // contributions lie inside the region
    for (int k = mt.z; k < k1; ++k) {
      const double* sb = S + k * 9;
#pragma unroll
      for (int i = 0; i < 9; ++i) blk[i] += sb[i];
    }
    const unsigned mc = (unsigned)mt.y;
    int rj = 0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (!(mn >> j & 1u)) continue;
      double* row = P.K + tg.x + (int64_t)rj * L;
      int rk = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (!(mc >> k & 1u)) continue;
        row[rk] = ACC ? row[rk] + blk[3 * j + k] : blk[3 * j + k];
        ++rk;
      }
      ++rj;
    }
    if (tg.y >= 0) {                             // the transpose into c's rows
      int rk = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (!(mc >> k & 1u)) continue;
        double* row = P.K + tg.y + (int64_t)rk * mt.x;
        int cj = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          if (!(mn >> j & 1u)) continue;
          row[cj] = ACC ? row[cj] + blk[3 * j + k] : blk[3 * j + k];
          ++cj;
        }
        ++rk;
      }
    } else if (WR) {                             // the residual, incidences in element order
      double r[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < nq; ++q) {
#pragma unroll
        for (int j = 0; j < 3; ++j) r[j] += SR[q * 4 + j];
      }
      double* Rout = P.R + rdn;
      int rr = 0;
#pragma unroll
      for (int j = 0; j < 3; ++j)
        if (mn >> j & 1u) {
          Rout[rr] = ACC ? Rout[rr] + r[j] : r[j];
          ++rr;
        }
    }
    u += LPN;                                    // rows of more upper blocks than the group has lanes
    if (u < nu) {
      const longlong2* rp = reinterpret_cast<const longlong2*>(P.ublk + u0 + u);
      tg = rp[0];
      mt = *reinterpret_cast<const int4*>(rp + 1);
    }
  }
}

// R-only kernel: one thread per node, sequential over its incidences.
template <int NN, bool ACC, bool ER>
__global__ void __launch_bounds__(128) k_vol_r(VolParams P) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  const unsigned mn = P.mask[n];
  if (!mn) return;
  double r[3] = {0.0, 0.0, 0.0};
  for (int q = P.nodeinc[n]; q < P.nodeinc[n + 1]; ++q) {
    const int ea = P.inc[q];
    const int64_t e = ea >> 4;
    const int a = ea & 15;
    int32_t cn[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
    double racc[3];
    element_strip<NN, false>(P, cn, a, nullptr, racc);
    if (ER) {
#pragma unroll
      for (int j = 0; j < 3; ++j) P.elemR[(int64_t)(3 * a + j) * P.ne + e] = racc[j];
    }
    r[0] += racc[0]; r[1] += racc[1]; r[2] += racc[2];
  }
  double* Rout = P.R + P.rdof[n];
  int rj = 0;
#pragma unroll
  for (int j = 0; j < 3; ++j)
    if (mn >> j & 1u) {
      if (ACC) Rout[rj] += r[j];
      else Rout[rj] = r[j];
      ++rj;
    }
}

// ---- element energy: thread per element, deterministic two-stage sum ----
template <int NN>
__global__ void __launch_bounds__(256) k_vol_energy(VolParams P, double* partial) {
  __shared__ double sh[256];
  const int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (e < P.ne) {
    int32_t cn[NN];
    unsigned mk[NN];
    int32_t rd[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      cn[b] = P.conn[e * NN + b];
      mk[b] = P.mask[cn[b]];
      rd[b] = P.rdof[cn[b]];
    }
#pragma unroll
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double w, F[9], iF[9], J, iJ[9];
      gauss_kin<NN>(P, cn, mk, rd, g, w, F, iF, J, iJ);
      double sF2 = 0.0;
#pragma unroll
      for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
      double I1 = sF2 * jm23(J);
      double W = P.mu / 2.0 * (I1 - 3.0) + P.kappa / 2.0 * (J - 1.0) * (J - 1.0);
      acc += W * w;
    }
  }
  double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ partial, int64_t n, double* out,
                                                      int accumulate) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 256) acc += partial[i];
  double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) out[0] = accumulate ? out[0] + s : s;
}

// ---- follower pressure (enclosed volume) ---------------------------------
struct FaceParams {
  const double* __restrict__ Xi;   // instance coordinates
  const int32_t* __restrict__ rdof;
  const uint8_t* __restrict__ mask;
  const int64_t* __restrict__ vbase;
  const int32_t* __restrict__ rowlen;
  const int32_t* __restrict__ dbase;
  const int32_t* __restrict__ conn;
  const int32_t* __restrict__ inc;
  const uint16_t* __restrict__ boff;
  const int32_t* __restrict__ nodeinc;
  const int32_t* __restrict__ chunkptr;
  const int32_t* __restrict__ chunkinc;
  const int32_t* __restrict__ chunklist;
  const int32_t* __restrict__ chunkdim;
  const int32_t* __restrict__ soff;
  const int32_t* __restrict__ roff;
  const double* __restrict__ gc;
  double* K;
  double* R;
  double p;
  int64_t nf;
  int32_t maxval;
};

template <int NF>
struct Face;
template <>
struct Face<3> {
  static constexpr int NG = 3;
  __device__ static __forceinline__ double sf(int g, int m, int a) { return c_sf_t3[g][m][a]; }
  __device__ static __forceinline__ double w(int g) { return c_w_t3[g]; }
};
template <>
struct Face<4> {
  static constexpr int NG = 4;
  __device__ static __forceinline__ double sf(int g, int m, int a) { return c_sf_q4[g][m][a]; }
  __device__ static __forceinline__ double w(int g) { return c_w_q4[g]; }
};

// Frame r[i][m] = sum_b sf[m][b] x_b[i] (columns: x, x_xi, x_eta) at Gauss point g.
template <int NF>
__device__ __forceinline__ void face_frame(const double (*x)[3], int g, double r[9]) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < NF; ++b) s += Face<NF>::sf(g, m, b) * x[b][i];
      r[3 * i + m] = s;
    }
}

template <int NF>
__device__ __forceinline__ void face_nodes(const FaceParams& P, const int32_t* cn, double (*x)[3]) {
#pragma unroll
  for (int b = 0; b < NF; ++b) {
    unsigned m = P.mask[cn[b]];
    int32_t rd = P.rdof[cn[b]];
#pragma unroll
    for (int i = 0; i < 3; ++i) x[b][i] = P.Xi[3 * (int64_t)cn[b] + i] + node_u(P.gc, rd, m, i);
  }
}

// Pressure.get_stiffness (pressure.py:80-132) for row node a of one face:
//   dV/dx_a[i]       = sum_g w/3 A_i,            A_i = sum_m sf[m][a] cof[i][m]
//   d2V/dx_a,i dx_b,j = sum_g w/3 (A_i C_j(b) - D_i(b) B_j),
//   B_j = sum_m sf[m][a] inv[m][j], C_j(b) = sum_n sf[n][b] inv[n][j],
//   D_i(b) = sum_n sf[n][b] cof[i][n], cof = det * inv^T.
// The assembly adds +p dV/dx to R and +p d2V/dx2 to K (assembly.py:336-341).
template <int NF>
__global__ void __launch_bounds__(128) k_face_rk(FaceParams P) {
  extern __shared__ double sm[];
  const int ch = blockIdx.x;
  const int i0 = P.chunkinc[ch], i1 = P.chunkinc[ch + 1];
  const int nv = P.chunkdim[3 * ch];
  const int nr = P.chunkdim[3 * ch + 1];
  for (int i = threadIdx.x; i < nv + nr; i += blockDim.x) sm[i] = 0.0;
  __syncthreads();
  const int q = i0 + threadIdx.x;
  const bool act = q < i1;
  double kacc[NF][9];
  double racc[3] = {0.0, 0.0, 0.0};
  int32_t cn[NF];
  int rank = -1, n = 0;
  unsigned mn = 0;
  int rowoff = 0, L = 0, dr = 0;
  if (act) {
    const int ea = P.inc[q];
    const int64_t f = ea >> 4;
    const int a = ea & 15;
#pragma unroll
    for (int b = 0; b < NF; ++b) cn[b] = P.conn[f * NF + b];
    n = cn[a];
    rank = q - P.nodeinc[n];
    mn = P.mask[n];                              // the row metadata, issued before the face math
    rowoff = P.soff[n];
    L = P.rowlen[n];
    dr = P.roff[n];
    double x[NF][3];
    face_nodes<NF>(P, cn, x);
#pragma unroll
    for (int b = 0; b < NF; ++b)
#pragma unroll
      for (int i = 0; i < 9; ++i) kacc[b][i] = 0.0;
#pragma unroll
    for (int g = 0; g < Face<NF>::NG; ++g) {
      double r[9], inv[9];
      face_frame<NF>(x, g, r);
      double det = inv3(r, inv);
      double w3 = Face<NF>::w(g) / 3.0 * P.p;
      double A[3], B[3];
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        double sa = 0.0, sb = 0.0;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          sa += Face<NF>::sf(g, m, a) * det * inv[3 * m + i];   // cof[i][m] = det inv[m][i]
          sb += Face<NF>::sf(g, m, a) * inv[3 * m + i];         // B_i
        }
        A[i] = sa;
        B[i] = sb;
      }
#pragma unroll
      for (int i = 0; i < 3; ++i) racc[i] += w3 * A[i];
#pragma unroll
      for (int b = 0; b < NF; ++b) {
        double C[3], D[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double sc = 0.0;
#pragma unroll
          for (int m = 0; m < 3; ++m) sc += Face<NF>::sf(g, m, b) * inv[3 * m + j];
          C[j] = sc;
          D[j] = det * sc;   // D_i(b) = sum_n sf[n][b] det inv[n][i]
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) kacc[b][3 * i + j] += w3 * (A[i] * C[j] - D[i] * B[j]);
      }
    }
  }
  for (int k = 0; k < P.maxval; ++k) {
    if (rank == k) {
      if (P.K) {
#pragma unroll
        for (int b = 0; b < NF; ++b) {
          const unsigned bo = P.boff[(int64_t)q * NF + b];
          if (bo == 0xFFFFu) continue;
          const unsigned mc = P.mask[cn[b]];
          int rj = 0;
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            if (!(mn >> j & 1u)) continue;
            double* row = sm + rowoff + rj * L + bo;
            int rk = 0;
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
              if (!(mc >> kk & 1u)) continue;
              row[rk] += kacc[b][3 * j + kk];
              ++rk;
            }
            ++rj;
          }
        }
      }
      if (P.R) {
        int rj = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
          if (mn >> j & 1u) sm[nv + dr + rj++] += racc[j];
      }
    }
    __syncthreads();
  }
  write_back<true>(P.chunkptr, P.chunklist, P.chunkdim, P.vbase, P.dbase, P.mask, P.soff, P.roff, ch, sm, P.K, nv, P.R);
}

template <int NF>
__global__ void __launch_bounds__(256) k_face_volume(FaceParams P, double* partial) {
  __shared__ double sh[256];
  const int64_t f = (int64_t)blockIdx.x * 256 + threadIdx.x;
  double acc = 0.0;
  if (f < P.nf) {
    int32_t cn[NF];
#pragma unroll
    for (int b = 0; b < NF; ++b) cn[b] = P.conn[f * NF + b];
    double x[NF][3];
    face_nodes<NF>(P, cn, x);
#pragma unroll
    for (int g = 0; g < Face<NF>::NG; ++g) {
      double r[9];
      face_frame<NF>(x, g, r);
      acc += Face<NF>::w(g) * det3(r) / 3.0;
    }
  }
  double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// ---- device line search -----------------------------------------------------
// The Armijo backtracking of the Newton solver (static_implicit.py:97-169)
// with its trial energies evaluated on the device: a ladder of LS_M trial
// steps alpha_k = 2^-(k0 + k) per launch, every element (and pressure face)
// evaluated at all of them in one pass, and the first step that passes the
// test selected and applied on the device.  The state vector (LS_*) carries
// the directional derivative, the energy at the current point, the largest
// step component, the direction's sign and the outcome.
constexpr int LS_M = 8;
enum { LS_DE = 0, LS_E0, LS_SMAX, LS_SIGN, LS_ALPHA, LS_ENEW, LS_FOUND, LS_ROUND, LS_NSTATE };

template <int NN>
__global__ void __launch_bounds__(128) k_vol_energy_ladder(VolParams P, const double* __restrict__ dgc,
                                                           const double* __restrict__ state, int k0,
                                                           double* __restrict__ partial, int64_t nb) {
  __shared__ double sh[128];
  const int64_t e = (int64_t)blockIdx.x * 128 + threadIdx.x;
  double acc[LS_M];
#pragma unroll
  for (int k = 0; k < LS_M; ++k) acc[k] = 0.0;
  if (e < P.ne) {
    int32_t cn[NN];
    unsigned mk[NN];
    int32_t rd[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      cn[b] = P.conn[e * NN + b];
      mk[b] = P.mask[cn[b]];
      rd[b] = P.rdof[cn[b]];
    }
    const double sgn = state[LS_SIGN];
#pragma unroll 1
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double J0[9], Ju[9], Jd[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) J0[i] = Ju[i] = Jd[i] = 0.0;
#pragma unroll
      for (int b = 0; b < NN; ++b) {
        const double* xb = P.X + 3 * (int64_t)cn[b];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const double x = __ldg(xb + i), u = node_u(P.gc, rd[b], mk[b], i), du = node_u(dgc, rd[b], mk[b], i);
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            const double d = Elem<NN>::dxi(g, b, m);
            J0[3 * i + m] += x * d;
            Ju[3 * i + m] += u * d;
            Jd[3 * i + m] += du * d;
          }
        }
      }
      double iJ[9];
      const double w = inv3(J0, iJ) * Elem<NN>::wq(g);
      double Gu[9], Gd[9];
#pragma unroll
      for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          Gu[3 * I + i] = (I == i ? 1.0 : 0.0) + Ju[3 * I] * iJ[i] + Ju[3 * I + 1] * iJ[3 + i] + Ju[3 * I + 2] * iJ[6 + i];
          Gd[3 * I + i] = Jd[3 * I] * iJ[i] + Jd[3 * I + 1] * iJ[3 + i] + Jd[3 * I + 2] * iJ[6 + i];
        }
#pragma unroll
      for (int k = 0; k < LS_M; ++k) {
        const double a = sgn * ldexp(1.0, -(k0 + k));
        double F[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) F[i] = Gu[i] + a * Gd[i];
        const double J = det3(F);
        double sF2 = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) sF2 += F[i] * F[i];
        const double I1 = sF2 * jm23(J);
        acc[k] += (P.mu / 2.0 * (I1 - 3.0) + P.kappa / 2.0 * (J - 1.0) * (J - 1.0)) * w;
      }
    }
  }
#pragma unroll 1
  for (int k = 0; k < LS_M; ++k) {
    const double s = block_sum<128>(acc[k], sh);
    if (threadIdx.x == 0) partial[k * nb + blockIdx.x] = s;
  }
}

template <int NF>
__global__ void __launch_bounds__(128) k_face_volume_ladder(FaceParams P, const double* __restrict__ dgc,
                                                            const double* __restrict__ state, int k0,
                                                            double* __restrict__ partial, int64_t nb) {
  __shared__ double sh[128];
  const int64_t f = (int64_t)blockIdx.x * 128 + threadIdx.x;
  double acc[LS_M];
#pragma unroll
  for (int k = 0; k < LS_M; ++k) acc[k] = 0.0;
  if (f < P.nf) {
    int32_t cn[NF];
#pragma unroll
    for (int b = 0; b < NF; ++b) cn[b] = P.conn[f * NF + b];
    double x[NF][3], d[NF][3];
    face_nodes<NF>(P, cn, x);
#pragma unroll
    for (int b = 0; b < NF; ++b) {
      const unsigned m = P.mask[cn[b]];
      const int32_t rd = P.rdof[cn[b]];
#pragma unroll
      for (int i = 0; i < 3; ++i) d[b][i] = node_u(dgc, rd, m, i);
    }
    const double sgn = state[LS_SIGN];
#pragma unroll
    for (int g = 0; g < Face<NF>::NG; ++g) {
      double rx[9], rd[9];
      face_frame<NF>(x, g, rx);
      face_frame<NF>(d, g, rd);
#pragma unroll
      for (int k = 0; k < LS_M; ++k) {
        const double a = sgn * ldexp(1.0, -(k0 + k));
        double r[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) r[i] = rx[i] + a * rd[i];
        acc[k] += Face<NF>::w(g) * det3(r) / 3.0;
      }
    }
  }
#pragma unroll 1
  for (int k = 0; k < LS_M; ++k) {
    const double s = block_sum<128>(acc[k], sh);
    if (threadIdx.x == 0) partial[k * nb + blockIdx.x] = s;
  }
}

// out[k] (+)= scale * sum_i partial[k * nb + i], fixed order; one block per k
__global__ void __launch_bounds__(256) k_sum_ladder(const double* __restrict__ partial, int64_t nb, double scale,
                                                    double* out, int accumulate) {
  __shared__ double sh[256];
  const int k = blockIdx.x;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < nb; i += 256) acc += partial[k * nb + i];
  const double s = block_sum<256>(acc, sh);
  if (threadIdx.x == 0) out[k] = (accumulate ? out[k] : 0.0) + scale * s;
}

// per-block sum of dgc.R and max |dgc|
__global__ void __launch_bounds__(256) k_ls_partial(int64_t n, const double* __restrict__ dgc,
                                                    const double* __restrict__ R, double* partial, int64_t nb) {
  __shared__ double sh[256];
  double dot = 0.0, mx = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
    const double d = dgc[i];
    dot += d * R[i];
    mx = fmax(mx, fabs(d));
  }
  const double s = block_sum<256>(dot, sh);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s;
    partial[nb + blockIdx.x] = sh[0];
  }
}

__global__ void __launch_bounds__(256) k_ls_prepare(const double* __restrict__ partial, int64_t nb,
                                                    const double* __restrict__ e0, double* state) {
  __shared__ double sh[256];
  double dot = 0.0, mx = 0.0;
  for (int64_t i = threadIdx.x; i < nb; i += 256) {
    dot += partial[i];
    mx = fmax(mx, partial[nb + i]);
  }
  const double de = block_sum<256>(dot, sh);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double E0 = e0[0];
    state[LS_SIGN] = de > 0.0 ? -1.0 : 1.0;      // the reference turns an ascent direction around
    state[LS_DE] = de > 0.0 ? -de : de;
    state[LS_E0] = E0;
    state[LS_SMAX] = sh[0];
    state[LS_ALPHA] = 0.0;
    state[LS_ENEW] = E0;
    state[LS_FOUND] = 0.0;
    // the predicted decrease is below the energy's own round-off: the
    // energy comparison carries no information (the host decides instead)
    state[LS_ROUND] = fabs(de) <= 1e-10 * fabs(E0) ? 1.0 : 0.0;
  }
}

// first accepted step of the ladder [k0, k0 + LS_M): Armijo with c1 and the
// step-length cap; alpha below 1e-12 ends the search without a step
__global__ void k_ls_select(const double* __restrict__ E, int k0, double c1, double max_step, double* state) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (state[LS_FOUND] != 0.0 || state[LS_ROUND] != 0.0) return;
  for (int k = 0; k < LS_M; ++k) {
    const double a = ldexp(1.0, -(k0 + k));
    if (a < 1e-12) {
      state[LS_FOUND] = -1.0;
      return;
    }
    const double e = E[k];
    const bool ok = isfinite(e) && e <= state[LS_E0] + c1 * state[LS_DE] * a && a * state[LS_SMAX] <= max_step;
    if (ok) {
      state[LS_ALPHA] = state[LS_SIGN] * a;
      state[LS_ENEW] = e;
      state[LS_FOUND] = 1.0;
      return;
    }
  }
}

// gc += alpha dgc once a step has been accepted
__global__ void __launch_bounds__(256) k_ls_apply(int64_t n, const double* __restrict__ state,
                                                  const double* __restrict__ dgc, double* gc) {
  if (state[LS_FOUND] != 1.0) return;
  const double a = state[LS_ALPHA];
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
    gc[i] += a * dgc[i];
}

// ---- lumped mass: thread per node ------------------------------------------
// m[(n,d)] += sum_{e,b} rho w N_a N_b over free (conn[e][b], d), the row sum
// of the reduced consistent mass (C3base.py:348-384, assembly.py:421-443,
// dynamic_explicit.py:147-167).
template <int NN>
__global__ void __launch_bounds__(128) k_lumped_mass(VolParams P, double rho, double* m) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  const unsigned mn = P.mask[n];
  if (!mn) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int q = P.nodeinc[n]; q < P.nodeinc[n + 1]; ++q) {
    const int ea = P.inc[q];
    const int64_t e = ea >> 4;
    const int a = ea & 15;
    int32_t cn[NN];
    unsigned mk[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      cn[b] = P.conn[e * NN + b];
      mk[b] = P.mask[cn[b]];
    }
#pragma unroll
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double J0[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) J0[i] = 0.0;
#pragma unroll
      for (int b = 0; b < NN; ++b)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          double d = Elem<NN>::dxi(g, b, m);
#pragma unroll
          for (int i = 0; i < 3; ++i) J0[3 * i + m] += P.X[3 * (int64_t)cn[b] + i] * d;
        }
      double w = det3(J0) * Elem<NN>::wq(g) * rho * Elem<NN>::N(g, a);
#pragma unroll
      for (int b = 0; b < NN; ++b) {
        double t = w * Elem<NN>::N(g, b);
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (mk[b] >> d & 1u) acc[d] += t;
      }
    }
  }
  double* out = m + P.rdof[n];
  int rj = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
    if (mn >> d & 1u) out[rj++] += acc[d];
}

// Consistent mass in the reduced CSR values: one thread per row node n,
// incidences in element order; M_ab = sum_g rho N_a N_b w detJ0 of every
// incident element goes to the entries ((n, d), (c_b, d)) of the DOFs d free
// at both nodes (the mass couples like directions only), added to Mv.
// Follows Element_3D.get_mass_matrix (C3base.py:348-384) with the reduction
// of Assembly.assemble_mass_matrix (assembly.py:421-443).
template <int NN>
__global__ void __launch_bounds__(128) k_mass_csr(VolParams P, double rho, double* __restrict__ Mv) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= P.n_nodes) return;
  const unsigned mn = P.mask[n];
  if (!mn) return;
  const int L = P.rowlen[n];
  const int64_t vb = P.vbase[n];
  for (int q = P.nodeinc[n]; q < P.nodeinc[n + 1]; ++q) {
    const int ea = P.inc[q];
    const int64_t e = ea >> 4;
    const int a = ea & 15;
    int32_t cn[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) cn[b] = P.conn[e * NN + b];
    double mab[NN];
#pragma unroll
    for (int b = 0; b < NN; ++b) mab[b] = 0.0;
#pragma unroll
    for (int g = 0; g < Elem<NN>::NG; ++g) {
      double J0[9];
#pragma unroll
      for (int i = 0; i < 9; ++i) J0[i] = 0.0;
#pragma unroll
      for (int b = 0; b < NN; ++b)
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          double d = Elem<NN>::dxi(g, b, m);
#pragma unroll
          for (int i = 0; i < 3; ++i) J0[3 * i + m] += P.X[3 * (int64_t)cn[b] + i] * d;
        }
      const double w = det3(J0) * Elem<NN>::wq(g) * rho * Elem<NN>::N(g, a);
#pragma unroll
      for (int b = 0; b < NN; ++b) mab[b] += w * Elem<NN>::N(g, b);
    }
#pragma unroll
    for (int b = 0; b < NN; ++b) {
      const unsigned bo = P.boff[(int64_t)q * NN + b];
      if (bo == 0xFFFFu) continue;                   // column node without free DOFs
      const unsigned mc = P.mask[cn[b]];
      int rd = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (!(mn >> d & 1u)) continue;
        if (mc >> d & 1u) Mv[vb + (int64_t)rd * L + bo + __popc(mc & ((1u << d) - 1u))] += mab[b];
        ++rd;
      }
    }
  }
}

__global__ void k_axpy(int64_t n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += alpha * x[i];
}

__global__ void k_invert_mass(int64_t n, double* m) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    double v = m[i];
    m[i] = 1.0 / (fabs(v) < 1e-12 ? 1.0 : v);
  }
}

// ---- host side ---------------------------------------------------------------
static VolParams vol_params(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                            const double* gc) {
  VolParams P;
  P.X = N->X_dev;
  P.rdof = N->rdof_dev;
  P.mask = N->mask_dev;
  P.vbase = N->vbase_dev;
  P.rowlen = N->rowlen_dev;
  P.dbase = N->dbase_dev;
  P.conn = G->conn_dev;
  P.inc = G->inc_dev;
  P.boff = G->boff_dev;
  P.nodeinc = G->nodeinc_dev;
  P.chunkptr = G->chunkptr_dev;
  P.chunkinc = G->chunkinc_dev;
  P.chunklist = G->chunklist_dev;
  P.chunkdim = G->chunkdim_dev;
  P.soff = G->soff_dev;
  P.roff = G->roff_dev;
  P.adjptr = N->adjptr_dev;
  P.adjcol = N->adjcol_dev;
  P.adjoff = N->adjoff_dev;
  P.uptr = G->uptr_dev;
  P.ublk = G->ublk_dev;
  P.incpos = G->incpos_dev;
  P.stagepos = G->stagepos_dev;
  P.region = G->region_dev;
  P.moff = N->moff_dev;
  P.gc = gc;
  P.K = P.R = P.elemR = nullptr;
  P.mu = mu;
  P.kappa = kappa;
  P.ne = G->ne;
  P.maxval = G->maxval;
  P.n_nodes = (int32_t)N->n_nodes;
  return P;
}

static int smem_limit() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

template <class Prm>
static int launch_chunked(void (*kern)(Prm), int64_t nchunk, int threads, int64_t smem_doubles, cudaStream_t st,
                          const Prm& p) {
  size_t bytes = (size_t)smem_doubles * sizeof(double);
  if (bytes > (size_t)smem_limit()) return FEA_ESMEM;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return (int)err;
  if (nchunk <= 0) return 0;
  kern<<<(unsigned)nchunk, threads, bytes, st>>>(p);
  count_launch();
  return (int)cudaGetLastError();
}

template <class Prm, class X>
static int launch_chunked_ex(void (*kern)(Prm, X), int64_t nchunk, int threads, int64_t smem_doubles,
                             cudaStream_t st, const Prm& p, X extra) {
  size_t bytes = (size_t)smem_doubles * sizeof(double);
  if (bytes > (size_t)smem_limit()) return FEA_ESMEM;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err != cudaSuccess) return (int)err;
  if (nchunk <= 0) return 0;
  kern<<<(unsigned)nchunk, threads, bytes, st>>>(p, extra);
  count_launch();
  return (int)cudaGetLastError();
}

}  // namespace fea

using namespace fea;

extern "C" int64_t fea_reduce_scratch_len(int64_t n_items) { return (n_items + 255) / 256 + 1; }

extern "C" int64_t fea_assemble_work_len(const fea_group_t* G) {
  if (!G || G->kind != FEA_C3D8) return 0;
  // residual slots: one per incidence, or maxval per node in the fixed layout
  const int64_t slots = G->hx_stride > 0 ? (G->nblk / G->hx_stride) * (int64_t)G->maxval : G->ne * 8;
  return hx_rslot_base(G->nblk) + slots * 4;
}

extern "C" int fea_assemble_volume(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                   const double* gc, double* K, double* R, double* elemR, int32_t accumulate,
                                   double* work, int64_t work_len, cudaStream_t st) {
  // gc may be NULL when no DOF is free (the kernels read it for free DOFs only)
  if (!N || !G || (!gc && N->ndof > 0) || (G->kind != FEA_C3D4 && G->kind != FEA_C3D8)) return FEA_EINVAL;
  if (G->nn != (G->kind == FEA_C3D8 ? 8 : 4)) return FEA_EINVAL;
  const bool hex = G->kind == FEA_C3D8;
  const int tpb = hex ? HX_GINC : VolTPB<4>::v;
  if (G->threads != tpb) return FEA_ECHUNK;
  // every argument check comes before the first device call
  if (K && hex) {
    // an empty group stages nothing (work length 0): its gather writes zero
    // blocks, or adds them, and reads neither work nor the element arrays
    const int64_t wneed = fea_assemble_work_len(G);
    if ((wneed > 0 && !work) || work_len < wneed) return FEA_EWORK;
    if (((uintptr_t)work & 15) != 0) return FEA_EINVAL;
    if (G->ne < 0 || (G->ne > 0 && (!G->incpos_dev || !G->stagepos_dev)) || !G->region_dev || !G->uptr_dev ||
        !G->ublk_dev || G->nblk < 0 || G->maxblk < 0)
      return FEA_EINVAL;
  }
  if (!K) {
    if (!R && !elemR) return FEA_OK;
    if (!R) return FEA_EINVAL;  // the residual-only path writes R
  }
  if (int r = ensure_tables()) return r;
  VolParams P = vol_params(N, G, mu, kappa, gc);
  P.K = K;
  P.R = R;
  P.elemR = elemR;
  if (K) {
    int64_t smem = G->smem_doubles;
    const bool acc = accumulate != 0, wr = R != nullptr, er = elemR != nullptr;
    if (hex) {
      const bool fixed = G->hx_stride > 0;
      if (fixed && G->hx_stride != G->maxblk) return FEA_EINVAL;
      const int capb = std::max<int>(G->maxblk, 2);   // regions hold even block counts
      const int capq = std::max<int>(G->maxval, 1);   // most incidences of one node
      const size_t region = ((size_t)capb * 9 + (wr ? (size_t)capq * 4 : 0)) * sizeof(double);
      const bool two = (size_t)HX_GW * (32 / HX_LPN) * region <= (size_t)smem_limit();
      const int lpn = two ? HX_LPN : 32;
      const size_t gbytes = (size_t)HX_GW * (32 / lpn) * region;
      if (gbytes > (size_t)smem_limit()) return FEA_ESMEM;
      double* rslot = work + hx_rslot_base(G->nblk);
      const unsigned grid = (unsigned)((G->ne + HX_EPB - 1) / HX_EPB);
      if (grid) {
        if (er) k_hex_elem<true><<<grid, HX_TPB, 0, st>>>(P, work, rslot);
        else k_hex_elem<false><<<grid, HX_TPB, 0, st>>>(P, work, rslot);
        count_launch();
        if (cudaError_t ce = cudaGetLastError()) return (int)ce;
      }
      const int per_cta = HX_GW * (32 / lpn);
      const unsigned g2 = (unsigned)((N->n_nodes + per_cta - 1) / per_cta);
      if (g2) {
        void (*gk)(VolParams, const double*, const double*, int, int) =
            fixed ? (two ? (wr ? (acc ? k_hex_gat<true, true, HX_LPN, true> : k_hex_gat<true, false, HX_LPN, true>)
                               : (acc ? k_hex_gat<false, true, HX_LPN, true> : k_hex_gat<false, false, HX_LPN, true>))
                         : (wr ? (acc ? k_hex_gat<true, true, 32, true> : k_hex_gat<true, false, 32, true>)
                               : (acc ? k_hex_gat<false, true, 32, true> : k_hex_gat<false, false, 32, true>)))
                  : (two ? (wr ? (acc ? k_hex_gat<true, true, HX_LPN, false> : k_hex_gat<true, false, HX_LPN, false>)
                               : (acc ? k_hex_gat<false, true, HX_LPN, false> : k_hex_gat<false, false, HX_LPN, false>))
                         : (wr ? (acc ? k_hex_gat<true, true, 32, false> : k_hex_gat<true, false, 32, false>)
                               : (acc ? k_hex_gat<false, true, 32, false> : k_hex_gat<false, false, 32, false>)));
        if (cudaError_t ce = cudaFuncSetAttribute(gk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gbytes))
          return (int)ce;
        gk<<<g2, HX_GW * 32, gbytes, st>>>(P, work, rslot, capb, capq);
        count_launch();
      }
      return (int)cudaGetLastError();
    }
#define FEA_RK(NN_, WR_, ACC_, ER_)                                                                    \
  if (wr == WR_ && acc == ACC_ && er == ER_)                                                           \
    return launch_chunked(k_vol_rk<NN_, WR_, ACC_, ER_>, G->nchunk, tpb, smem, st, P);
    FEA_RK(4, true, false, false) FEA_RK(4, true, true, false) FEA_RK(4, false, false, false)
    FEA_RK(4, false, true, false) FEA_RK(4, true, false, true) FEA_RK(4, true, true, true)
    FEA_RK(4, false, false, true) FEA_RK(4, false, true, true)
#undef FEA_RK
    return FEA_EINVAL;
  }
  const int grid = grid_for(N->n_nodes, 128);
  if (N->n_nodes == 0) return FEA_OK;
  if (hex) {
    if (accumulate) elemR ? k_vol_r<8, true, true><<<grid, 128, 0, st>>>(P) : k_vol_r<8, true, false><<<grid, 128, 0, st>>>(P);
    else elemR ? k_vol_r<8, false, true><<<grid, 128, 0, st>>>(P) : k_vol_r<8, false, false><<<grid, 128, 0, st>>>(P);
  } else {
    if (accumulate) elemR ? k_vol_r<4, true, true><<<grid, 128, 0, st>>>(P) : k_vol_r<4, true, false><<<grid, 128, 0, st>>>(P);
    else elemR ? k_vol_r<4, false, true><<<grid, 128, 0, st>>>(P) : k_vol_r<4, false, false><<<grid, 128, 0, st>>>(P);
  }
  count_launch();
  return (int)cudaGetLastError();
}

static FaceParams face_params(const fea_nodes_t* N, const fea_group_t* G, double p, const double* Xi,
                              const double* gc) {
  FaceParams P;
  P.Xi = Xi;
  P.rdof = N->rdof_dev;
  P.mask = N->mask_dev;
  P.vbase = N->vbase_dev;
  P.rowlen = N->rowlen_dev;
  P.dbase = N->dbase_dev;
  P.conn = G->conn_dev;
  P.inc = G->inc_dev;
  P.boff = G->boff_dev;
  P.nodeinc = G->nodeinc_dev;
  P.chunkptr = G->chunkptr_dev;
  P.chunkinc = G->chunkinc_dev;
  P.chunklist = G->chunklist_dev;
  P.chunkdim = G->chunkdim_dev;
  P.soff = G->soff_dev;
  P.roff = G->roff_dev;
  P.gc = gc;
  P.K = P.R = nullptr;
  P.p = p;
  P.nf = G->ne;
  P.maxval = G->maxval;
  return P;
}

extern "C" int fea_assemble_pressure(const fea_nodes_t* N, const fea_group_t* G, double p, const double* Xi,
                                     const double* gc, double* K, double* R, cudaStream_t st) {
  if (!N || !G || !Xi || (!gc && N->ndof > 0) || (G->kind != FEA_T3 && G->kind != FEA_Q4)) return FEA_EINVAL;
  if (G->nn != (G->kind == FEA_T3 ? 3 : 4) || (G->threads != 32 && G->threads != 128)) return FEA_EINVAL;
  if (!K && !R) return FEA_OK;
  if (int r = ensure_tables()) return r;
  FaceParams P = face_params(N, G, p, Xi, gc);
  P.K = K;
  P.R = R;
  if (G->kind == FEA_T3) return launch_chunked(k_face_rk<3>, G->nchunk, G->threads, G->smem_doubles, st, P);
  return launch_chunked(k_face_rk<4>, G->nchunk, G->threads, G->smem_doubles, st, P);
}

extern "C" int fea_energy_volume(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                 const double* gc, double* out, double* scratch, int64_t scratch_len,
                                 cudaStream_t st) {
  if (!N || !G || (!gc && N->ndof > 0) || !out || !scratch) return FEA_EINVAL;
  if (G->kind != FEA_C3D4 && G->kind != FEA_C3D8) return FEA_EINVAL;
  if (scratch_len < fea_reduce_scratch_len(G->ne)) return FEA_EWORK;
  if (int r = ensure_tables()) return r;
  VolParams P = vol_params(N, G, mu, kappa, gc);
  const int64_t nb = (G->ne + 255) / 256;
  if (nb > 0) {
    if (G->kind == FEA_C3D8) k_vol_energy<8><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    else k_vol_energy<4><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    count_launch();
  }
  k_sum_partials<<<1, 256, 0, st>>>(scratch, nb, out, 0);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_energy_pressure(const fea_nodes_t* N, const fea_group_t* G, const double* Xi,
                                   const double* gc, double* out, double* scratch, int64_t scratch_len,
                                   cudaStream_t st) {
  if (!N || !G || !Xi || (!gc && N->ndof > 0) || !out || !scratch) return FEA_EINVAL;
  if (G->kind != FEA_T3 && G->kind != FEA_Q4) return FEA_EINVAL;
  if (scratch_len < fea_reduce_scratch_len(G->ne)) return FEA_EWORK;
  if (int r = ensure_tables()) return r;
  FaceParams P = face_params(N, G, 0.0, Xi, gc);
  const int64_t nb = (G->ne + 255) / 256;
  if (nb > 0) {
    if (G->kind == FEA_T3) k_face_volume<3><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    else k_face_volume<4><<<(unsigned)nb, 256, 0, st>>>(P, scratch);
    count_launch();
  }
  k_sum_partials<<<1, 256, 0, st>>>(scratch, nb, out, 0);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_lumped_mass(const fea_nodes_t* N, const fea_group_t* G, double rho, double* m,
                               cudaStream_t st) {
  if (!N || !G || !m || (G->kind != FEA_C3D4 && G->kind != FEA_C3D8)) return FEA_EINVAL;
  if (int r = ensure_tables()) return r;
  if (N->n_nodes == 0) return FEA_OK;
  VolParams P = vol_params(N, G, 0.0, 0.0, nullptr);
  const int grid = grid_for(N->n_nodes, 128);
  if (G->kind == FEA_C3D8) k_lumped_mass<8><<<grid, 128, 0, st>>>(P, rho, m);
  else k_lumped_mass<4><<<grid, 128, 0, st>>>(P, rho, m);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_mass_csr(const fea_nodes_t* N, const fea_group_t* G, double rho, double* Mv,
                            cudaStream_t st) {
  if (!N || !G || !Mv || (G->kind != FEA_C3D4 && G->kind != FEA_C3D8) || !G->boff_dev) return FEA_EINVAL;
  if (int r = ensure_tables()) return r;
  if (N->n_nodes == 0) return FEA_OK;
  VolParams P = vol_params(N, G, 0.0, 0.0, nullptr);
  const int grid = grid_for(N->n_nodes, 128);
  if (G->kind == FEA_C3D8) k_mass_csr<8><<<grid, 128, 0, st>>>(P, rho, Mv);
  else k_mass_csr<4><<<grid, 128, 0, st>>>(P, rho, Mv);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_axpy(int64_t n, double alpha, const double* x, double* y, cudaStream_t st) {
  if (n < 0 || (n > 0 && (!x || !y))) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  const int64_t g = std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_axpy<<<(unsigned)g, 256, 0, st>>>(n, alpha, x, y);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_invert_mass(int64_t n, double* m, cudaStream_t st) {
  if (!m || n < 0) return FEA_EINVAL;
  if (n == 0) return FEA_OK;
  k_invert_mass<<<grid_for(n, 256), 256, 0, st>>>(n, m);
  count_launch();
  return (int)cudaGetLastError();
}

// ---- allocation-free element energy ----------------------------------------
// Same kernels and reduction order as fea_energy_volume, but the per-block
// partial sums live in a fixed array that is part of this library's device
// image instead of a caller-provided buffer.  It exists for callers that
// cannot allocate device memory at the point of the call: hosts that hand all
// device memory to their own pool allocator up front, or foreign-language
// hosts that only pass pointers they already own.
static constexpr int64_t kNoallocMaxElems = FEA_NOALLOC_MAX_ELEMS;
static __device__ __align__(256) double g_noalloc_partials[(kNoallocMaxElems + 255) / 256];
static std::atomic<double*> g_noalloc_ptr[64];   // device address of the array, per device ordinal

extern "C" int fea_energy_volume_noalloc(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                         const double* gc, double* out, cudaStream_t st) {
  if (!N || !G || !gc || !out) return FEA_EINVAL;
  if (G->kind != FEA_C3D4 && G->kind != FEA_C3D8) return FEA_EINVAL;
  if (G->ne < 0) return FEA_EINVAL;
  if (G->ne > kNoallocMaxElems) return FEA_ETOOBIG;
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev)) return (int)e;
  if (dev < 0 || dev >= 64) return FEA_EINVAL;
  double* part = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!part) {
    // host code cannot use the array's name as a device address: resolve it
    // once per device, with that device current
    void* p = nullptr;
    if (cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials)) return (int)e;
    part = static_cast<double*>(p);
    g_noalloc_ptr[dev].store(part, std::memory_order_release);
  }
  if (int r = ensure_tables()) return r;
  VolParams P = vol_params(N, G, mu, kappa, gc);
  const int64_t nb = (G->ne + 255) / 256;
  if (nb > 0) {
    if (G->kind == FEA_C3D8) k_vol_energy<8><<<(unsigned)nb, 256, 0, st>>>(P, part);
    else k_vol_energy<4><<<(unsigned)nb, 256, 0, st>>>(P, part);
    count_launch();
  }
  k_sum_partials<<<1, 256, 0, st>>>(part, nb, out, 0);
  count_launch();
  return (int)cudaGetLastError();
}

// ---- device line search entry points ------------------------------------------
extern "C" int32_t fea_ls_ladder_len() { return LS_M; }

extern "C" int64_t fea_ls_scratch_len(int64_t n_items) { return (int64_t)LS_M * ((n_items + 127) / 128) + 16; }

extern "C" int fea_ls_energy_volume(const fea_nodes_t* N, const fea_group_t* G, double mu, double kappa,
                                    const double* gc, const double* dgc, const double* state, int32_t k0,
                                    int32_t accumulate, double* out, double* scratch, int64_t scratch_len,
                                    cudaStream_t st) {
  if (!N || !G || !gc || !dgc || !state || !out || !scratch || k0 < 0) return FEA_EINVAL;
  if (G->kind != FEA_C3D4 && G->kind != FEA_C3D8) return FEA_EINVAL;
  if (scratch_len < fea_ls_scratch_len(G->ne)) return FEA_EWORK;
  if (int r = ensure_tables()) return r;
  VolParams P = vol_params(N, G, mu, kappa, gc);
  const int64_t nb = (G->ne + 127) / 128;
  if (nb > 0) {
    if (G->kind == FEA_C3D8) k_vol_energy_ladder<8><<<(unsigned)nb, 128, 0, st>>>(P, dgc, state, k0, scratch, nb);
    else k_vol_energy_ladder<4><<<(unsigned)nb, 128, 0, st>>>(P, dgc, state, k0, scratch, nb);
    count_launch();
  }
  k_sum_ladder<<<LS_M, 256, 0, st>>>(scratch, nb, 1.0, out, accumulate);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_ls_energy_pressure(const fea_nodes_t* N, const fea_group_t* G, double p, const double* Xi,
                                      const double* gc, const double* dgc, const double* state, int32_t k0,
                                      int32_t accumulate, double* out, double* scratch, int64_t scratch_len,
                                      cudaStream_t st) {
  if (!N || !G || !Xi || !gc || !dgc || !state || !out || !scratch || k0 < 0) return FEA_EINVAL;
  if (G->kind != FEA_T3 && G->kind != FEA_Q4) return FEA_EINVAL;
  if (scratch_len < fea_ls_scratch_len(G->ne)) return FEA_EWORK;
  if (int r = ensure_tables()) return r;
  FaceParams P = face_params(N, G, p, Xi, gc);
  const int64_t nb = (G->ne + 127) / 128;
  if (nb > 0) {
    if (G->kind == FEA_T3) k_face_volume_ladder<3><<<(unsigned)nb, 128, 0, st>>>(P, dgc, state, k0, scratch, nb);
    else k_face_volume_ladder<4><<<(unsigned)nb, 128, 0, st>>>(P, dgc, state, k0, scratch, nb);
    count_launch();
  }
  k_sum_ladder<<<LS_M, 256, 0, st>>>(scratch, nb, p, out, accumulate);
  count_launch();
  return (int)cudaGetLastError();
}

extern "C" int fea_ls_prepare(int64_t n, const double* dgc, const double* R, const double* e0, double* state,
                              double* scratch, int64_t scratch_len, cudaStream_t st) {
  if (n < 0 || !dgc || !R || !e0 || !state || !scratch) return FEA_EINVAL;
  const int64_t nb = n > 0 ? std::min<int64_t>((n + 255) / 256, 1024) : 1;
  if (scratch_len < 2 * nb) return FEA_EWORK;
  k_ls_partial<<<(unsigned)nb, 256, 0, st>>>(n, dgc, R, scratch, nb);
  k_ls_prepare<<<1, 256, 0, st>>>(scratch, nb, e0, state);
  count_launch(2);
  return (int)cudaGetLastError();
}

extern "C" int fea_ls_select(int64_t n, const double* E, int32_t k0, double c1, double max_step, double* state,
                             const double* dgc, double* gc, cudaStream_t st) {
  if (n < 0 || !E || !state || !dgc || !gc || k0 < 0) return FEA_EINVAL;
  k_ls_select<<<1, 32, 0, st>>>(E, k0, c1, max_step, state);
  const int64_t nb = n > 0 ? std::min<int64_t>((n + 255) / 256, 4096) : 1;
  k_ls_apply<<<(unsigned)nb, 256, 0, st>>>(n, state, dgc, gc);
  count_launch(2);
  return (int)cudaGetLastError();
}
