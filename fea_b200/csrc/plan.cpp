// Host-side assembly plan: reduced DOF numbering, node adjacency, reduced CSR
// pattern and the per-node gather lists used by the element kernels.
//
// Replaces, once per mesh, the reference's sort-based COO pattern and
// element-to-slot map (FEA/assemble/elements/C3/C3base.py:109-153) and the
// per-Newton-iteration Dirichlet masking + unique() relabelling
// (FEA/assemble/assembly.py:357-387).  The resulting CSR (indptr, indices)
// is, by construction, the coalesced reduced pattern of the reference:
// rows/cols are free DOFs in node-major order (GC order, assembly.py:170-183)
// and a row (n, j) holds every free DOF (c, k) of every node c sharing an
// element or a pressure face with n, sorted by column.
//
// The element-to-slot map is kept at node level: for every (row node n,
// incident element e) pair the plan stores, per element node b, the offset
// of node conn[e][b]'s column block inside row n (uint16).  The value of
// K[(n,j),(c,k)] lives at vbase[n] + rank(j)*rowlen[n] + boff + rank(k).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "../../include/fea_b200.h"

namespace {

inline int popc3(uint8_t m) { return (m & 1) + ((m >> 1) & 1) + ((m >> 2) & 1); }

int nodes_per(int kind) {
  switch (kind) {
    case FEA_C3D4: return 4;
    case FEA_C3D8: return 8;
    case FEA_T3: return 3;
    case FEA_Q4: return 4;
    default: return -1;
  }
}

struct GatherList {            // one element group or one face group
  int kind = 0, nn = 0;
  int64_t ne = 0;
  std::vector<int32_t> inc;      // e*16 + a
  std::vector<uint16_t> boff;    // [ninc, nn]
  std::vector<int32_t> nodeinc;  // [N+1]
  std::vector<int32_t> chunklist;  // nodes with incidences, chunk by chunk
  std::vector<int32_t> chunkptr;   // [nchunk+1] into chunklist
  std::vector<int32_t> chunkinc;   // [nchunk+1] first incidence
  std::vector<int32_t> chunkdim;   // [nchunk*3]: values, residual entries, contiguous flag
  std::vector<int32_t> soff;       // [N] shared-memory offset of the node's values in its chunk
  std::vector<int32_t> roff;       // [N] offset of its residual entries (after the chunk's values)
  std::vector<int64_t> uptr;       // [N+1] first upper-block record of each node (C3D8)
  std::vector<int64_t> ublk;       // [nu*4] upper-block records, fea_ublk_t layout
  std::vector<int32_t> incpos;     // [ne*nn] incidence index of (e, a), -1 for a node without rows
  std::vector<int32_t> stagepos;   // [ne*36] staged block of each element block (lane slot order), -1: none
  std::vector<int64_t> region;     // [N+1] first staged block of each node's region (even)
  int32_t hx_stride = 0;           // C3D8: regions at n * hx_stride, 16 records per node (0: by region / uptr)
  std::vector<int32_t> allptr;     // [N+1] incidences of every node (constrained ones included)
  std::vector<int32_t> allinc;     // e*16 + a, element order ascending
  int64_t maxval = 0, threads = 0, smem = 0;
};

template <class F>
void parallel_for(int64_t n, F f) {
  unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  if (n < 4096 || hw == 1) { f(0, n); return; }
  std::vector<std::thread> th;
  int64_t step = (n + hw - 1) / hw;
  for (unsigned t = 0; t < hw; ++t) {
    int64_t a = t * step, b = std::min<int64_t>(n, a + step);
    if (a >= b) break;
    th.emplace_back([=, &f] { f(a, b); });
  }
  for (auto& t : th) t.join();
}

}  // namespace

struct fea_plan {
  int64_t N = 0, ndof = 0, nnz = 0, nnzb = 0;
  std::vector<int32_t> rdof, dbase, rowlen;
  std::vector<uint8_t> mask;
  std::vector<int64_t> vbase, indptr, adjptr;
  std::vector<int32_t> indices, adjcol, adjoff;
  std::vector<int32_t> moff;       // [nnzb] value offset of n in row c, for entry (n, c)
  std::vector<GatherList> groups, faces;
};

namespace {

// node -> incident (element, local index) lists, element order ascending
struct Incidence {
  std::vector<int64_t> ptr;   // [N+1]
  std::vector<int64_t> ent;   // e*16 + a
};

int build_incidence(int64_t N, int nn, int64_t ne, const int32_t* conn, Incidence& inc) {
  inc.ptr.assign(N + 1, 0);
  for (int64_t i = 0; i < ne * nn; ++i) {
    int32_t v = conn[i];
    if (v < 0 || v >= N) return FEA_ERANGE;
    inc.ptr[v + 1]++;
  }
  for (int64_t n = 0; n < N; ++n) inc.ptr[n + 1] += inc.ptr[n];
  inc.ent.resize(inc.ptr[N]);
  std::vector<int64_t> fill(inc.ptr.begin(), inc.ptr.end() - 1);
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < nn; ++a) inc.ent[fill[conn[e * nn + a]]++] = e * 16 + a;
  return FEA_OK;
}

int build_gather(const fea_plan& P, int kind, int64_t ne, const int32_t* conn, const Incidence& I,
                 int threads, int64_t smem_budget, GatherList& G) {
  G.kind = kind;
  G.nn = nodes_per(kind);
  G.ne = ne;
  const int nn = G.nn;
  const int64_t N = P.N;
  G.nodeinc.assign(N + 1, 0);
  for (int64_t n = 0; n < N; ++n) {
    int64_t c = P.mask[n] ? (I.ptr[n + 1] - I.ptr[n]) : 0;
    G.nodeinc[n + 1] = (int32_t)(G.nodeinc[n] + c);
    G.maxval = std::max<int64_t>(G.maxval, c);
  }
  int64_t ninc = G.nodeinc[N];
  if (ninc >= INT32_MAX) return FEA_ERANGE;
  G.inc.resize(ninc);
  G.boff.resize(ninc * nn);
  int err = FEA_OK;
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    for (int64_t n = a0; n < a1; ++n) {
      if (!P.mask[n]) continue;
      int64_t o = G.nodeinc[n];
      const int32_t* col = P.adjcol.data() + P.adjptr[n];
      int64_t ncol = P.adjptr[n + 1] - P.adjptr[n];
      for (int64_t q = I.ptr[n]; q < I.ptr[n + 1]; ++q, ++o) {
        int64_t e = I.ent[q] >> 4;
        G.inc[o] = (int32_t)I.ent[q];
        for (int b = 0; b < nn; ++b) {
          int32_t c = conn[e * nn + b];
          uint16_t bo = 0xFFFF;
          if (P.mask[c]) {
            const int32_t* it = std::lower_bound(col, col + ncol, c);
            if (it == col + ncol || *it != c) { err = FEA_ERANGE; continue; }
            int32_t off = P.adjoff[P.adjptr[n] + (it - col)];
            if (off >= 0xFFFF) { err = FEA_ECHUNK; continue; }
            bo = (uint16_t)off;
          }
          G.boff[o * nn + b] = bo;
        }
      }
    }
  });
  if (err) return err;
  G.incpos.assign((size_t)ne * nn, -1);
  for (int64_t o = 0; o < ninc; ++o) G.incpos[(size_t)(G.inc[o] >> 4) * nn + (G.inc[o] & 15)] = (int32_t)o;
  // chunks of nodes that have incidences in this list (in node order):
  // incidences <= threads, shared doubles <= budget
  G.allptr.assign(N + 1, 0);
  for (int64_t n = 0; n < N; ++n) G.allptr[n + 1] = (int32_t)I.ptr[n + 1];
  G.allinc.resize(I.ent.size());
  for (size_t i = 0; i < I.ent.size(); ++i) G.allinc[i] = (int32_t)I.ent[i];
  G.threads = threads;
  G.soff.assign(N, 0);
  G.roff.assign(N, 0);
  G.chunkptr.push_back(0);
  G.chunkinc.push_back(0);
  std::vector<int32_t> cur;
  int64_t cur_inc = 0, cur_v = 0, cur_r = 0;
  auto close = [&]() {
    if (cur.empty()) return;
    int32_t r = 0;
    bool contig = true;
    for (size_t i = 0; i < cur.size(); ++i) {
      int32_t n = cur[i];
      G.roff[n] = r;
      r += popc3(P.mask[n]);
      if (i + 1 < cur.size()) {
        int32_t m = cur[i + 1];
        if (P.vbase[n + 1] != P.vbase[m] || P.dbase[n + 1] != P.dbase[m]) contig = false;
      }
    }
    for (int32_t n : cur) G.chunklist.push_back(n);
    G.chunkptr.push_back((int32_t)G.chunklist.size());
    G.chunkinc.push_back(G.nodeinc[cur.back() + 1]);
    G.chunkdim.push_back((int32_t)cur_v);
    G.chunkdim.push_back((int32_t)cur_r);
    G.chunkdim.push_back(contig ? 1 : 0);
    G.smem = std::max(G.smem, cur_v + cur_r);
    cur.clear();
    cur_inc = cur_v = cur_r = 0;
  };
  for (int64_t n = 0; n < N; ++n) {
    int64_t ni = G.nodeinc[n + 1] - G.nodeinc[n];
    if (ni == 0) continue;
    int64_t f = popc3(P.mask[n]);
    int64_t v = f * (int64_t)P.rowlen[n];
    // the C3D8 kernels read no chunks (staged blocks and a node-row gather
    // instead): a node of more incidences than a chunk takes gets a chunk of
    // its own there, and only the C3D4 and face lists are bounded
    if (kind != FEA_C3D8 && (ni > threads || v + f > smem_budget)) return FEA_ECHUNK;
    if (cur_inc + ni > threads || cur_v + v + cur_r + f > smem_budget) close();
    if (!cur.empty() && G.nodeinc[cur.back() + 1] != G.nodeinc[n]) close();
    G.soff[n] = (int32_t)cur_v;
    cur.push_back((int32_t)n);
    cur_inc += ni;
    cur_v += v;
    cur_r += f;
  }
  close();
  return FEA_OK;
}

// Staging of a C3D8 group.  An element block couples the unordered local
// pair {i, j} (36 per element: 8 diagonal, 28 off-diagonal) and belongs to
// the upper node block (r, c), r = min(n_i, n_j), c = max(n_i, n_j), when both
// nodes are active.  The element kernel's lane a computes K_ab for b = (a +
// d) & 7, d = 0..3 and d = 4 for a < 4: the owner slot of {i, j}.  A node's
// region lists, block-major, the contributions to each of its upper blocks
// (adjacency order, c >= r; a block may have none), each block's in ascending
// element order (then ascending slot, for an element that repeats a node);
// regions start at even block indices (16-byte aligned).  stagepos maps
// (e, slot) to the contribution's staged block; the upper-block records give
// the gather its targets and contributor range.
int owner_slot(int i, int j) {
  int a = i, d = (j - i) & 7;
  if (!(d < 4 || (d == 4 && i < 4))) {
    a = j;
    d = (i - j) & 7;
  }
  return (a < 4 ? 5 * a : 20 + 4 * (a - 4)) + d;
}

int build_blocks(const fea_plan& P, int nn, const int32_t* conn, const Incidence& I, GatherList& G) {
  const int64_t N = P.N;
  // contribution of incidence (e, i) of node r with local node j: the pair
  // {i, j} counted once, from its lower-numbered node (from i <= j when the
  // element repeats the node)
  auto contributes = [&](int64_t e, int i, int j, int32_t r) {
    const int32_t c = conn[e * nn + j];
    return P.mask[c] && (c > r || (c == r && j >= i));
  };
  std::vector<int32_t> cnt(P.nnzb, 0);
  int err = FEA_OK;
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    for (int64_t n = a0; n < a1; ++n) {
      if (!P.mask[n]) continue;
      const int32_t* col = P.adjcol.data() + P.adjptr[n];
      const int64_t ncol = P.adjptr[n + 1] - P.adjptr[n];
      for (int64_t q = I.ptr[n]; q < I.ptr[n + 1]; ++q) {
        const int64_t e = I.ent[q] >> 4;
        const int i = (int)(I.ent[q] & 15);
        for (int j = 0; j < nn; ++j) {
          if (!contributes(e, i, j, (int32_t)n)) continue;
          const int32_t c = conn[e * nn + j];
          const int32_t* it = std::lower_bound(col, col + ncol, c);
          if (it == col + ncol || *it != c) { err = FEA_ERANGE; continue; }
          cnt[P.adjptr[n] + (it - col)]++;
        }
      }
    }
  });
  if (err) return err;
  G.region.assign(N + 1, 0);
  G.uptr.assign(N + 1, 0);
  int64_t smax = 0, umax = 0;
  for (int64_t n = 0; n < N; ++n) {
    int64_t nb = 0, nu = 0;
    if (P.mask[n])
      for (int64_t p = P.adjptr[n]; p < P.adjptr[n + 1]; ++p)
        if (P.adjcol[p] >= n) {
          nb += cnt[p];
          ++nu;
        }
    nb = (nb + 1) & ~(int64_t)1;
    smax = std::max(smax, nb);
    umax = std::max(umax, nu);
    G.region[n + 1] = G.region[n] + nb;
    G.uptr[n + 1] = G.uptr[n] + nu;
  }
  // Regular meshes (a structured block: 36 blocks in an interior region)
  // take a fixed stride, so that the gather can start a node's region copy
  // and record loads without first loading where they are: regions at
  // n * smax, 16 record slots per node (unused ones with row = -1), the
  // residual slots of node n at n * maxval.  Chosen when it costs at most a
  // quarter more staging than the packed layout.
  G.hx_stride = 0;
  // (residual slots are addressed n * maxval in 32 bits)
  if (smax > 0 && umax <= 16 && smax <= 96 && N * smax <= G.region[N] + G.region[N] / 4 &&
      N * (int64_t)G.maxval < INT32_MAX) {
    G.hx_stride = (int32_t)smax;
    for (int64_t n = 0; n <= N; ++n) {
      G.region[n] = n * smax;
      G.uptr[n] = n * 16;
    }
  }
  if (G.region[N] >= INT32_MAX) return FEA_ERANGE;
  G.ublk.assign((size_t)G.uptr[N] * 4, 0);
  if (G.hx_stride)
    for (int64_t u = 0; u < G.uptr[N]; ++u) G.ublk[4 * u] = G.ublk[4 * u + 1] = -1;   // unused slots
  G.stagepos.assign((size_t)G.ne * 36, -1);
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    std::vector<int64_t> fill;
    for (int64_t n = a0; n < a1; ++n) {
      if (!P.mask[n]) continue;
      const int64_t p0 = P.adjptr[n], np = P.adjptr[n + 1] - p0;
      const int32_t* col = P.adjcol.data() + p0;
      fill.assign(np, -1);
      int64_t t = 0, u = G.uptr[n];
      for (int64_t k = 0; k < np; ++k) {
        const int32_t c = col[k];
        if (c < n) continue;
        fill[k] = t;
        int64_t* rec = G.ublk.data() + 4 * u++;
        rec[0] = P.vbase[n] + P.adjoff[p0 + k];
        rec[1] = c != n ? P.vbase[c] + P.moff[p0 + k] : -1;
        rec[2] = (int64_t)(uint32_t)P.rowlen[c] | ((int64_t)P.mask[c] << 32);
        rec[3] = (int64_t)(uint32_t)t | ((int64_t)cnt[p0 + k] << 32);
        t += cnt[p0 + k];
      }
      for (int64_t q = I.ptr[n]; q < I.ptr[n + 1]; ++q) {
        const int64_t e = I.ent[q] >> 4;
        const int i = (int)(I.ent[q] & 15);
        for (int j = 0; j < nn; ++j) {
          if (!contributes(e, i, j, (int32_t)n)) continue;
          const int64_t k = std::lower_bound(col, col + np, conn[e * nn + j]) - col;
          G.stagepos[e * 36 + owner_slot(i, j)] = (int32_t)(G.region[n] + fill[k]++);
        }
      }
    }
  });
  if (G.hx_stride) {
    // residual slot of incidence (e, a) of node n: n * maxval + its rank
    for (int64_t n = 0; n < N; ++n)
      for (int32_t q = G.nodeinc[n]; q < G.nodeinc[n + 1]; ++q) {
        const int32_t ea = G.inc[q];
        G.incpos[(size_t)(ea >> 4) * nn + (ea & 15)] = (int32_t)(n * G.maxval + (q - G.nodeinc[n]));
      }
  }
  return FEA_OK;
}

}  // namespace

extern "C" int fea_plan_build(int64_t n_nodes, const uint8_t* free_mask, int32_t n_groups,
                              const int32_t* group_kind, const int64_t* group_ne,
                              const int32_t* const* group_conn, int32_t n_faces, const int32_t* face_kind,
                              const int64_t* face_nf, const int32_t* const* face_conn, int32_t vol_threads,
                              int64_t smem_doubles, fea_plan** out) {
  if (!out || n_nodes < 0 || n_nodes >= INT32_MAX || (n_nodes > 0 && !free_mask) || n_groups < 0 ||
      n_faces < 0)
    return FEA_EINVAL;
  *out = nullptr;
  for (int g = 0; g < n_groups; ++g) {
    int k = group_kind[g];
    if ((k != FEA_C3D4 && k != FEA_C3D8) || group_ne[g] < 0 || (group_ne[g] > 0 && !group_conn[g]))
      return FEA_EINVAL;
  }
  for (int g = 0; g < n_faces; ++g) {
    int k = face_kind[g];
    if ((k != FEA_T3 && k != FEA_Q4) || face_nf[g] < 0 || (face_nf[g] > 0 && !face_conn[g])) return FEA_EINVAL;
  }
  // incidences are coded e * 16 + a in 32 bits
  for (int g = 0; g < n_groups; ++g)
    if (group_ne[g] > FEA_PLAN_MAX_ELEMS) return FEA_ETOOBIG;
  for (int g = 0; g < n_faces; ++g)
    if (face_nf[g] > FEA_PLAN_MAX_ELEMS) return FEA_ETOOBIG;
  std::unique_ptr<fea_plan> P(new fea_plan);
  const int64_t N = n_nodes;
  P->N = N;
  P->mask.assign(free_mask, free_mask + N);
  for (auto& m : P->mask) m &= 7;
  // free-DOF numbering (node-major)
  P->dbase.assign(N + 1, 0);
  P->rdof.assign(N, -1);
  for (int64_t n = 0; n < N; ++n) {
    int f = popc3(P->mask[n]);
    if (f) P->rdof[n] = P->dbase[n];
    if ((int64_t)P->dbase[n] + f >= INT32_MAX) return FEA_ERANGE;
    P->dbase[n + 1] = P->dbase[n] + f;
  }
  P->ndof = P->dbase[N];
  // incidences
  std::vector<Incidence> ginc(n_groups), finc(n_faces);
  for (int g = 0; g < n_groups; ++g) {
    int r = build_incidence(N, nodes_per(group_kind[g]), group_ne[g], group_conn[g], ginc[g]);
    if (r) return r;
  }
  for (int g = 0; g < n_faces; ++g) {
    int r = build_incidence(N, nodes_per(face_kind[g]), face_nf[g], face_conn[g], finc[g]);
    if (r) return r;
  }
  // node adjacency over active nodes (sorted neighbour lists)
  std::vector<std::vector<int32_t>> adj(N);
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    std::vector<int32_t> tmp;
    for (int64_t n = a0; n < a1; ++n) {
      if (!P->mask[n]) continue;
      tmp.clear();
      auto add = [&](const Incidence& I, int nn, const int32_t* conn) {
        for (int64_t q = I.ptr[n]; q < I.ptr[n + 1]; ++q) {
          int64_t e = I.ent[q] >> 4;
          for (int b = 0; b < nn; ++b) {
            int32_t c = conn[e * nn + b];
            if (P->mask[c]) tmp.push_back(c);
          }
        }
      };
      for (int g = 0; g < n_groups; ++g) add(ginc[g], nodes_per(group_kind[g]), group_conn[g]);
      for (int g = 0; g < n_faces; ++g) add(finc[g], nodes_per(face_kind[g]), face_conn[g]);
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      adj[n] = tmp;
    }
  });
  P->adjptr.assign(N + 1, 0);
  P->rowlen.assign(N, 0);
  P->vbase.assign(N + 1, 0);
  for (int64_t n = 0; n < N; ++n) {
    int64_t L = 0;
    for (int32_t c : adj[n]) L += popc3(P->mask[c]);
    if (L >= INT32_MAX) return FEA_ERANGE;
    P->rowlen[n] = (int32_t)L;
    P->adjptr[n + 1] = P->adjptr[n] + (int64_t)adj[n].size();
    P->vbase[n + 1] = P->vbase[n] + popc3(P->mask[n]) * L;
  }
  P->nnzb = P->adjptr[N];
  P->nnz = P->vbase[N];
  P->adjcol.resize(P->nnzb);
  P->adjoff.resize(P->nnzb);
  P->indptr.assign(P->ndof + 1, 0);
  P->indices.resize(P->nnz);
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    for (int64_t n = a0; n < a1; ++n) {
      int64_t o = P->adjptr[n];
      int32_t off = 0;
      for (int32_t c : adj[n]) {
        P->adjcol[o] = c;
        P->adjoff[o] = off;
        off += popc3(P->mask[c]);
        ++o;
      }
      int f = popc3(P->mask[n]);
      int64_t L = P->rowlen[n];
      for (int r = 0; r < f; ++r) {
        int64_t row = P->dbase[n] + r;
        int64_t v = P->vbase[n] + r * L;
        P->indptr[row] = v;
        for (int32_t c : adj[n]) {
          int32_t d = P->dbase[c];
          for (int k = 0; k < 3; ++k)
            if (P->mask[c] >> k & 1) P->indices[v++] = d++;
        }
      }
    }
  });
  P->indptr[P->ndof] = P->nnz;
  { std::vector<std::vector<int32_t>>().swap(adj); }
  // mirrored offsets: for entry (n, c), the value offset of n in row c
  P->moff.assign(P->nnzb, -1);
  int merr = FEA_OK;
  parallel_for(N, [&](int64_t a0, int64_t a1) {
    for (int64_t n = a0; n < a1; ++n)
      for (int64_t p = P->adjptr[n]; p < P->adjptr[n + 1]; ++p) {
        const int32_t c = P->adjcol[p];
        const int32_t* col = P->adjcol.data() + P->adjptr[c];
        const int64_t ncol = P->adjptr[c + 1] - P->adjptr[c];
        const int32_t* it = std::lower_bound(col, col + ncol, (int32_t)n);
        if (it == col + ncol || *it != n) { merr = FEA_ERANGE; continue; }
        P->moff[p] = P->adjoff[P->adjptr[c] + (it - col)];
      }
  });
  if (merr) return merr;
  // gather lists
  P->groups.resize(n_groups);
  P->faces.resize(n_faces);
  const int64_t budget = smem_doubles > 0 ? smem_doubles : 12288;
  for (int g = 0; g < n_groups; ++g) {
    int th = vol_threads > 0 ? vol_threads : (group_kind[g] == FEA_C3D8 ? 32 : 256);
    int r = build_gather(*P, group_kind[g], group_ne[g], group_conn[g], ginc[g], th, budget, P->groups[g]);
    if (r) return r;
    if (group_kind[g] == FEA_C3D8 && (r = build_blocks(*P, 8, group_conn[g], ginc[g], P->groups[g]))) return r;
  }
  for (int g = 0; g < n_faces; ++g) {
    // chunks of 32 face incidences (one warp per CTA: many small CTAs for the
    // few thousand faces of a loaded surface), 128 when a node has more
    int64_t most = 0;
    for (int64_t n = 0; n < N; ++n) most = std::max<int64_t>(most, finc[g].ptr[n + 1] - finc[g].ptr[n]);
    const int th = most <= 32 ? 32 : 128;
    int r = build_gather(*P, face_kind[g], face_nf[g], face_conn[g], finc[g], th, budget, P->faces[g]);
    if (r) return r;
  }
  *out = P.release();
  return FEA_OK;
}

extern "C" void fea_plan_free(fea_plan* plan) { delete plan; }

namespace {
template <class T>
int put(const std::vector<T>& v, void* dst, int64_t* count) {
  if (count) *count = (int64_t)v.size();
  if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(T));
  return FEA_OK;
}
int scalar(int64_t s, int64_t* count) {
  if (!count) return FEA_EINVAL;
  *count = s;
  return FEA_OK;
}
}  // namespace

extern "C" int fea_plan_get(const fea_plan* P, int32_t id, int32_t group, void* dst, int64_t* count) {
  if (!P) return FEA_EINVAL;
  const GatherList* G = nullptr;
  if (id >= 30 && id < 50) {
    if (group < 0 || group >= (int)P->groups.size()) return FEA_EINVAL;
    G = &P->groups[group];
    id -= 30;
  } else if (id >= 50 && id < 70) {
    if (group < 0 || group >= (int)P->faces.size()) return FEA_EINVAL;
    G = &P->faces[group];
    id -= 50;
  } else if (id >= 70 && id < 80) {               // element-group ids, continued
    if (group < 0 || group >= (int)P->groups.size()) return FEA_EINVAL;
    G = &P->groups[group];
    id -= 50;
  }
  if (G) {
    switch (id) {
      case 0: return put(G->inc, dst, count);
      case 1: return put(G->boff, dst, count);
      case 2: return put(G->nodeinc, dst, count);
      case 3: return put(G->chunkptr, dst, count);
      case 4: return put(G->chunkinc, dst, count);
      case 5: return scalar((int64_t)G->chunkptr.size() - 1, count);
      case 6: return scalar(G->maxval, count);
      case 7: return scalar(G->threads, count);
      case 8: return scalar(G->smem, count);
      case 9: return put(G->chunklist, dst, count);
      case 10: return put(G->chunkdim, dst, count);
      case 11: return put(G->soff, dst, count);
      case 12: return put(G->roff, dst, count);
      case 13: return put(G->uptr, dst, count);
      case 14: return put(G->ublk, dst, count);
      case 15: return put(G->allptr, dst, count);
      case 16: return put(G->allinc, dst, count);
      case 17: return put(G->incpos, dst, count);
      case 18: return put(G->stagepos, dst, count);
      case 19: return put(G->region, dst, count);
      case 20: return scalar(G->hx_stride, count);
      default: return FEA_EINVAL;
    }
  }
  switch (id) {
    case FEA_S_NDOF: return scalar(P->ndof, count);
    case FEA_S_NNZ: return scalar(P->nnz, count);
    case FEA_S_NNZB: return scalar(P->nnzb, count);
    case FEA_A_RDOF: return put(P->rdof, dst, count);
    case FEA_A_MASK: return put(P->mask, dst, count);
    case FEA_A_DBASE: return put(P->dbase, dst, count);
    case FEA_A_VBASE: return put(P->vbase, dst, count);
    case FEA_A_ROWLEN: return put(P->rowlen, dst, count);
    case FEA_A_INDPTR: return put(P->indptr, dst, count);
    case FEA_A_INDICES: return put(P->indices, dst, count);
    case FEA_A_ADJPTR: return put(P->adjptr, dst, count);
    case FEA_A_ADJCOL: return put(P->adjcol, dst, count);
    case FEA_A_ADJOFF: return put(P->adjoff, dst, count);
    case FEA_A_MOFF: return put(P->moff, dst, count);
    default: return FEA_EINVAL;
  }
}
