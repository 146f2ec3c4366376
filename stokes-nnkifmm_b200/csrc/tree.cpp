// Host octree + interaction lists + NEAREST source entries (see tree.h).
//
// Build with -ffp-contract=off: the midpoints and the NEAREST distances must
// round exactly like the reference's separate FP64 operations.
#include "tree.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>

#include "../../include/nnkifmm.h"
#include "common.h"

namespace nnk {

namespace {

struct Key3 {
  uint64_t a, b, c;
  bool operator==(const Key3& o) const { return a == o.a && b == o.b && c == o.c; }
};
inline uint64_t bits(double v) {
  v = v + 0.0;  // -0.0 -> +0.0: MATLAB compares rows by value
  uint64_t u;
  std::memcpy(&u, &v, 8);
  return u;
}
inline Key3 key(const double* p) { return Key3{bits(p[0]), bits(p[1]), bits(p[2])}; }

// The SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014) as a bit mixer.
inline uint64_t mix64(uint64_t x) {
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Point ids keyed by their rows in `pts` (bit patterns, -0.0 == +0.0), open
// addressing with linear probing.  insert() may run on many threads at once
// while `pts` does not change.
class PointTable {
 public:
  PointTable(int64_t expected, const std::vector<double>& pts) : pts_(pts) {
    size_t cap = 16;
    while (cap < (size_t)expected * 2) cap <<= 1;
    slots_.assign(cap, -1);
    mask_ = cap - 1;
  }
  // Inserts point id (its row is already in pts) unless an equal row is
  // present; returns the id that holds the row.
  int64_t insert(int64_t id) {
    const Key3 k = key(&pts_[3 * id]);
    size_t h = (size_t)mix64(k.a ^ mix64(k.b ^ mix64(k.c))) & mask_;
    for (;;) {
      int64_t cur = __atomic_load_n(&slots_[h], __ATOMIC_ACQUIRE);
      if (cur < 0 && __atomic_compare_exchange_n(&slots_[h], &cur, id, false, __ATOMIC_ACQ_REL,
                                                 __ATOMIC_ACQUIRE))
        return id;
      // cur: the id in the slot (a failed exchange loads it)
      if (key(&pts_[3 * cur]) == k) return cur;
      h = (h + 1) & mask_;
    }
  }

 private:
  const std::vector<double>& pts_;
  std::vector<int64_t> slots_;
  size_t mask_ = 0;
};

struct Builder {
  HostTree& t;
  std::string& msg;
  int err = 0;
  std::vector<int64_t> tmp;  // scratch for the counting sort

  // Dividenode (OcTree.m:181-222)
  void divide_node(int32_t node) {
    const double* c = &t.corners[6 * node];
    const double lo[3] = {c[0], c[1], c[2]};
    const double hi[3] = {c[3], c[4], c[5]};
    double ctr[3];
    for (int d = 0; d < 3; ++d) ctr[d] = (lo[d] + hi[d]) / 2.0;  // mean([lo;hi],1)
    const int64_t s = t.pstart[node], m = t.pcount[node];
    int64_t cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    tmp.resize(m);
    std::vector<uint8_t> oct(m);
    for (int64_t k = 0; k < m; ++k) {
      const double* p = &t.pts[3 * t.order[s + k]];
      int o = 4 * (p[0] > ctr[0]) + 2 * (p[1] > ctr[1]) + (p[2] > ctr[2]);
      oct[k] = (uint8_t)o;
      cnt[o]++;
    }
    int64_t off[8];
    off[0] = 0;
    for (int o = 1; o < 8; ++o) off[o] = off[o - 1] + cnt[o - 1];
    int64_t pos[8];
    std::memcpy(pos, off, sizeof(pos));
    for (int64_t k = 0; k < m; ++k) tmp[pos[oct[k]]++] = t.order[s + k];  // stable
    std::memcpy(&t.order[s], tmp.data(), m * sizeof(int64_t));
    const int32_t first = t.nodes;
    t.child0[node] = first;
    for (int o = 0; o < 8; ++o) {
      const int bx = (o >> 2) & 1, by = (o >> 1) & 1, bz = o & 1;
      const int32_t id = first + o;
      t.level.push_back(t.level[node] + 1);
      t.parent.push_back(node);
      t.child0.push_back(-1);
      t.ix.push_back(2 * t.ix[node] + bx);
      t.iy.push_back(2 * t.iy[node] + by);
      t.iz.push_back(2 * t.iz[node] + bz);
      const double nc[6] = {bx ? ctr[0] : lo[0], by ? ctr[1] : lo[1], bz ? ctr[2] : lo[2],
                            bx ? hi[0] : ctr[0], by ? hi[1] : ctr[1], bz ? hi[2] : ctr[2]};
      t.corners.insert(t.corners.end(), nc, nc + 6);
      t.pstart.push_back(s + off[o]);
      t.pcount.push_back(cnt[o]);
      (void)id;
    }
    t.nodes += 8;
  }

  // Divide (OcTree.m:155-179): the depth check runs for every visited node.
  void divide(int32_t b, int32_t e) {
    for (int32_t node = b; node < e && !err; ++node) {
      if (t.level[node] + 1 >= t.params.max_depth) {
        err = NNK_E_MAXDEPTH;
        msg = "Max level reached: Increase Max Depth";
        return;
      }
      const int32_t old = t.nodes;
      if (t.pcount[node] > t.capacity) {
        divide_node(node);
        divide(old, t.nodes);
      }
    }
  }
};

}  // namespace

bool HostTree::touch(int32_t a, int32_t b) const {
  const double* c1 = &corners[6 * a];
  const double* c2 = &corners[6 * b];
  return !(c2[0] > c1[3] || c2[3] < c1[0] || c2[1] > c1[4] || c2[4] < c1[1] ||
           c2[2] > c1[5] || c2[5] < c1[2]);
}

static void build_lists(HostTree& t) {
  const int32_t N = t.nodes;
  // colleagues, top-down
  t.colleagues.assign(N, {});
  t.colleagues[0].push_back(0);
  for (int L = 1; L <= t.max_level; ++L) {
    const std::vector<int32_t>& lv = t.by_level[L];
    const int64_t nl = (int64_t)lv.size();
    // nodes of one level are independent (they read their parents' lists)
#pragma omp parallel for schedule(static) if (nl > 2048)
    for (int64_t j = 0; j < nl; ++j) {
      const int32_t c = lv[j];
      const int32_t P = t.parent[c];
      auto& out = t.colleagues[c];
      for (int32_t C : t.colleagues[P]) {
        if (t.child0[C] < 0) continue;
        for (int k = 0; k < 8; ++k) {
          const int32_t cand = t.child0[C] + k;
          if (t.touch(c, cand)) out.push_back(cand);
        }
      }
      std::sort(out.begin(), out.end());
    }
  }
  // full: subtree without empty-potential leaves (bottom-up)
  t.full.assign(N, 0);
  for (int L = t.max_level; L >= 0; --L) {
    for (int32_t n : t.by_level[L]) {
      if (t.child0[n] < 0) {
        t.full[n] = t.pleaf[n];
      } else {
        uint8_t f = 1;
        for (int k = 0; k < 8; ++k) f &= t.full[t.child0[n] + k];
        t.full[n] = f;
      }
    }
  }

  std::vector<std::vector<int32_t>> U(N), V(N), W(N);
  // every node's lists are independent of the others'
#pragma omp parallel if (N > 2048)
  {
  std::vector<int32_t> stack;
#pragma omp for schedule(dynamic, 64)
  for (int32_t i = 1; i < N; ++i) {
    // V (OcTree.m:330-339): children of the parent's non-leaf same-level
    // touching nodes (other than the parent) that do not touch i.
    {
      const int32_t P = t.parent[i];
      auto& v = V[i];
      for (int32_t C : t.colleagues[P]) {
        if (C == P || t.child0[C] < 0) continue;
        for (int k = 0; k < 8; ++k) {
          const int32_t c = t.child0[C] + k;
          if (!t.touch(c, i)) v.push_back(c);
        }
      }
      std::sort(v.begin(), v.end());
    }
    if (!t.tleaf[i]) continue;
    // U (OcTree.m:323-327): every non-empty potential leaf touching i.
    {
      auto& u = U[i];
      for (int32_t a = i; a >= 0; a = t.parent[a]) {
        for (int32_t C : t.colleagues[a])
          if (t.child0[C] < 0 && t.pleaf[C] && t.touch(C, i)) u.push_back(C);
      }
      for (int32_t C : t.colleagues[i]) {
        if (t.child0[C] < 0) continue;
        stack.clear();
        for (int k = 0; k < 8; ++k) stack.push_back(t.child0[C] + k);
        while (!stack.empty()) {
          const int32_t n = stack.back();
          stack.pop_back();
          if (!t.touch(n, i)) continue;
          if (t.child0[n] < 0) {
            if (t.pleaf[n]) u.push_back(n);
          } else {
            for (int k = 0; k < 8; ++k) stack.push_back(t.child0[n] + k);
          }
        }
      }
      std::sort(u.begin(), u.end());
    }
    // W (OcTree.m:343-361): non-empty potential leaves below non-leaf
    // same-level touching nodes that do not touch i, with every complete
    // sibling block merged into its parent, bottom-up.  A subtree that does
    // not touch i merges all the way up iff it holds no empty-potential leaf.
    {
      auto& w = W[i];
      int32_t last = -1;
      for (int32_t C : t.colleagues[i]) {
        if (t.child0[C] < 0) continue;
        stack.clear();
        for (int k = 0; k < 8; ++k) stack.push_back(t.child0[C] + k);
        while (!stack.empty()) {
          const int32_t n = stack.back();
          stack.pop_back();
          const bool leaf = t.child0[n] < 0;
          if (!t.touch(n, i)) {
            if (t.full[n]) {
              w.push_back(n);
              if (!leaf) {
                if (last < 0 || t.level[n] < t.level[last] ||
                    (t.level[n] == t.level[last] && n > last))
                  last = n;
              }
              continue;
            }
          }
          if (!leaf)
            for (int k = 0; k < 8; ++k) stack.push_back(t.child0[n] + k);
        }
      }
      std::sort(w.begin(), w.end());
      // Each merge is W = [setdiff(W,children); node]: W ends sorted except
      // for the last merged node (lowest level, then largest id), at the end.
      if (last >= 0) {
        w.erase(std::find(w.begin(), w.end(), last));
        w.push_back(last);
      }
    }
  }
  }
  auto to_csr = [&](std::vector<std::vector<int32_t>>& L, Csr& out) {
    out.off.assign(N + 1, 0);
    for (int32_t i = 0; i < N; ++i) out.off[i + 1] = out.off[i] + (int64_t)L[i].size();
    out.idx.resize(out.off[N]);
    for (int32_t i = 0; i < N; ++i)
      std::copy(L[i].begin(), L[i].end(), out.idx.begin() + out.off[i]);
  };
  to_csr(U, t.U);
  to_csr(V, t.V);
  to_csr(W, t.W);
  // X (OcTree.m:279-288): find(Wpadded == i) is column-major, so X(i) is
  // ordered by the position of i inside W(j), then by j.
  {
    struct E { int32_t i, pos, j; };
    std::vector<E> ent;
    ent.reserve(t.W.idx.size());
    for (int32_t j = 0; j < N; ++j)
      for (int64_t k = t.W.off[j]; k < t.W.off[j + 1]; ++k)
        ent.push_back({t.W.idx[k], (int32_t)(k - t.W.off[j]), j});
    std::sort(ent.begin(), ent.end(), [](const E& a, const E& b) {
      if (a.i != b.i) return a.i < b.i;
      if (a.pos != b.pos) return a.pos < b.pos;
      return a.j < b.j;
    });
    t.X.off.assign(N + 1, 0);
    for (auto& e : ent) t.X.off[e.i + 1]++;
    for (int32_t i = 0; i < N; ++i) t.X.off[i + 1] += t.X.off[i];
    t.X.idx.resize(ent.size());
    for (size_t k = 0; k < ent.size(); ++k) t.X.idx[k] = ent[k].j;
  }
}

int build_tree(const double* pot, int64_t n_pot, const double* tgt, int64_t n_tgt,
               const double* fine, int64_t q, const int64_t* nn_rowptr,
               const int32_t* nn_col, const double* nn_val, const TreeParams& p,
               HostTree& t, std::string& msg, struct ::nnk_ctx* gpu) {
  t = HostTree();
  t.params = p;
  if (n_pot < 0 || n_tgt < 0 || (n_pot && !pot) || (n_tgt && !tgt)) {
    msg = "invalid point arrays";
    return NNK_E_ARG;
  }
  if (p.max_depth > 23) {
    msg = "maxDepth above 23 is not supported";
    return NNK_E_ARG;
  }
  for (int64_t i = 0; i < 3 * n_pot; ++i)
    if (!std::isfinite(pot[i])) { msg = "non-finite potential point"; return NNK_E_NONFINITE; }
  for (int64_t i = 0; i < 3 * n_tgt; ++i)
    if (!std::isfinite(tgt[i])) { msg = "non-finite target point"; return NNK_E_NONFINITE; }
  const bool same = (pot == tgt && n_pot == n_tgt);
  if (p.nearest && !same) {
    msg = "NEAREST mode needs targetPoints == potPoints";
    return NNK_E_ARG;
  }
  // points = unique([pot;tgt],'rows','stable'); masks by ismember (OcTree.m:80-82)
  {
    // potPoints rows must be distinct, so they are points 0..n_pot-1
    t.pts.reserve(3 * (size_t)(n_pot + (same ? 0 : n_tgt)));
    t.pts.assign(pot, pot + 3 * n_pot);
    PointTable seen(n_pot + (same ? 0 : n_tgt), t.pts);
    int dup = 0;
#pragma omp parallel for schedule(static) reduction(| : dup) if (n_pot > 65536)
    for (int64_t i = 0; i < n_pot; ++i) dup |= (seen.insert(i) != i);
    if (dup) {
      msg = "potPoints contains duplicate rows";
      return NNK_E_ARG;
    }
    t.n = n_pot;
    std::vector<int64_t> pot_pt(n_pot);
    for (int64_t i = 0; i < n_pot; ++i) pot_pt[i] = i;
    std::vector<int64_t> tgt_pt;
    if (!same) {
      // targets in order: a new row becomes the next point
      tgt_pt.resize(n_tgt);
      for (int64_t i = 0; i < n_tgt; ++i) {
        t.pts.insert(t.pts.end(), tgt + 3 * i, tgt + 3 * i + 3);
        const int64_t id = seen.insert(t.n);
        if (id == t.n) {
          t.n++;
        } else {
          t.pts.resize(3 * t.n);
        }
        tgt_pt[i] = id;
      }
    }
    t.is_pot.assign(t.n, 0);
    t.is_tgt.assign(t.n, 0);
    for (int64_t i = 0; i < n_pot; ++i) t.is_pot[pot_pt[i]] = 1;
    if (same) {
      for (int64_t i = 0; i < n_pot; ++i) t.is_tgt[pot_pt[i]] = 1;
    } else {
      for (int64_t i = 0; i < n_tgt; ++i) t.is_tgt[tgt_pt[i]] = 1;
    }
    t.pot_rank.assign(t.n, -1);
    t.tgt_rank.assign(t.n, -1);
    for (int64_t i = 0; i < t.n; ++i) {
      if (t.is_pot[i]) t.pot_rank[i] = t.n_pot++;
      if (t.is_tgt[i]) t.tgt_rank[i] = t.n_tgt++;
    }
  }
  if (t.n < 1) {
    msg = "no points";
    return NNK_E_ARG;
  }
  // root cube (OcTree.m:97-98) and capacity (:105)
  double lo = t.pts[0], hi = t.pts[0];
  for (double v : t.pts) {
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  t.capacity = (int)std::min<int64_t>(p.node_capacity, t.n - 1);
  t.nodes = 1;
  t.level = {0};
  t.parent = {-1};
  t.child0 = {-1};
  t.ix = {0};
  t.iy = {0};
  t.iz = {0};
  t.corners = {lo, lo, lo, hi, hi, hi};
  t.order.resize(t.n);
  for (int64_t i = 0; i < t.n; ++i) t.order[i] = i;
  t.pstart = {0};
  t.pcount = {t.n};
  if (gpu) {
    const int rc = build_nodes_gpu(gpu, t, msg);
    if (rc) return rc;
  } else {
    Builder b{t, msg};
    b.divide(0, 1);
    if (b.err) return b.err;
  }
  const int32_t N = t.nodes;
  t.max_level = 0;
  for (int32_t i = 0; i < N; ++i) t.max_level = std::max(t.max_level, t.level[i]);
  t.by_level.assign(t.max_level + 1, {});
  for (int32_t i = 0; i < N; ++i) t.by_level[t.level[i]].push_back(i);
  t.point_index.assign(t.n, -1);
  t.tleaf.assign(N, 0);
  t.pleaf.assign(N, 0);
  for (int32_t i = 0; i < N; ++i) {
    if (t.child0[i] >= 0) continue;
    for (int64_t k = t.pstart[i]; k < t.pstart[i] + t.pcount[i]; ++k) {
      const int64_t pt = t.order[k];
      t.point_index[pt] = i;
      if (t.is_tgt[pt]) t.tleaf[i] = 1;
      if (t.is_pot[pt]) t.pleaf[i] = 1;
    }
  }
  if (gpu) build_lists_gpu(gpu, t);
  else build_lists(t);

  // ---- targets sorted by leaf (downwardPass.m:297-305 scatter order)
  t.tgt_start.assign(N + 1, 0);
  t.tgt_row.clear();
  t.tgt_pos.clear();
  for (int32_t i = 0; i < N; ++i) {
    t.tgt_start[i] = (int64_t)t.tgt_row.size();
    if (t.child0[i] < 0) {
      for (int64_t k = t.pstart[i]; k < t.pstart[i] + t.pcount[i]; ++k) {
        const int64_t pt = t.order[k];
        if (!t.is_tgt[pt]) continue;
        t.tgt_row.push_back((int32_t)t.tgt_rank[pt]);
        t.tgt_pos.insert(t.tgt_pos.end(), &t.pts[3 * pt], &t.pts[3 * pt] + 3);
      }
    }
  }
  t.tgt_start[N] = (int64_t)t.tgt_row.size();

  // ---- NEAREST matrix
  if (p.nearest) {
    if (q <= 0 || !fine) {
      msg = "NEAREST mode needs finePoints";
      return NNK_E_ARG;
    }
    for (int64_t i = 0; i < 3 * q; ++i)
      if (!std::isfinite(fine[i])) { msg = "non-finite fine point"; return NNK_E_NONFINITE; }
    t.q = q;
    t.fine.assign(fine, fine + 3 * q);
    if (nn_rowptr) {
      t.nn_rowptr.assign(nn_rowptr, nn_rowptr + q + 1);
      const int64_t nnz = t.nn_rowptr[q];
      // rowptr first: 0, non-decreasing, so every row lies inside [0, nnz)
      if (t.nn_rowptr[0] != 0 || nnz < 0) { msg = "bad NN rowptr"; return NNK_E_ARG; }
      for (int64_t r = 0; r < q; ++r)
        if (t.nn_rowptr[r + 1] < t.nn_rowptr[r]) { msg = "bad NN rowptr"; return NNK_E_ARG; }
      if (nnz > 0 && (!nn_col || !nn_val)) { msg = "NN columns or values missing"; return NNK_E_ARG; }
      t.nn_col.assign(nn_col, nn_col + nnz);
      t.nn_val.assign(nn_val, nn_val + nnz);
      int bad = 0;
      int32_t* col = t.nn_col.data();
      double* val = t.nn_val.data();
      const int64_t* rp = t.nn_rowptr.data();
#pragma omp parallel for schedule(static) reduction(| : bad) if (q > 65536)
      for (int64_t r = 0; r < q; ++r) {
        const int64_t a = rp[r], b = rp[r + 1];
        int row_bad = 0;
        for (int64_t k = a; k < b; ++k) row_bad |= (col[k] < 0 || col[k] >= n_pot);
        bad |= row_bad;
        if (row_bad) continue;
        // columns ascending within the row (MATLAB sparse storage order), by
        // (column, weight) like a sort of the pairs; rows hold a handful of
        // tied neighbours, so insertion sort
        for (int64_t k = a + 1; k < b; ++k) {
          const int32_t c = col[k];
          const double v = val[k];
          int64_t j = k;
          while (j > a && (col[j - 1] > c || (col[j - 1] == c && val[j - 1] > v))) {
            col[j] = col[j - 1];
            val[j] = val[j - 1];
            --j;
          }
          col[j] = c;
          val[j] = v;
        }
      }
      if (bad) { msg = "NN column out of range"; return NNK_E_ARG; }
    } else if (gpu) {
      nearest_matrix_gpu(gpu, pot, n_pot, fine, q, t.nn_rowptr, t.nn_col, t.nn_val);
    } else {
      nearest_matrix(pot, n_pot, fine, q, t.nn_rowptr, t.nn_col, t.nn_val);
    }
  }

  // ---- leaf source entries
  t.src_start.assign(N + 1, 0);
  t.src_pos.clear();
  t.src_goff.assign(1, 0);
  t.src_gidx.clear();
  t.src_gw.clear();
  t.src_origin.clear();
  if (!p.nearest) {
    // plain: potential points of each leaf (upwardPass.m:54-77)
    for (int32_t i = 0; i < N; ++i) {
      t.src_start[i] = (int64_t)t.src_goff.size() - 1;
      if (t.child0[i] >= 0) continue;
      for (int64_t k = t.pstart[i]; k < t.pstart[i] + t.pcount[i]; ++k) {
        const int64_t pt = t.order[k];
        if (!t.is_pot[pt]) continue;
        t.src_pos.insert(t.src_pos.end(), &t.pts[3 * pt], &t.pts[3 * pt] + 3);
        t.src_gidx.push_back((int32_t)t.pot_rank[pt]);
        t.src_gw.push_back(1.0);
        t.src_origin.push_back(t.pot_rank[pt]);
        t.src_goff.push_back((int64_t)t.src_gidx.size());
      }
    }
    t.src_start[N] = (int64_t)t.src_goff.size() - 1;
  } else {
    // NEAREST: fine points with a nonzero NN entry in the leaf's columns,
    // ascending fine index, each carrying kron(NN_sub,I3)*f
    // (upwardPass.m:58-66, downwardPass.m:89-101).
    struct T { int64_t q; int32_t col; double w; };
    std::vector<int64_t> cnt(N + 1, 0);
    const int64_t nnz = t.nn_rowptr[q];
    for (int64_t k = 0; k < nnz; ++k) {
      if (t.nn_val[k] == 0.0) continue;
      cnt[t.point_index[t.nn_col[k]] + 1]++;
    }
    for (int32_t i = 0; i < N; ++i) cnt[i + 1] += cnt[i];
    const int64_t G = cnt[N];
    // NN entries bucketed by leaf, ascending fine index inside a bucket
    std::vector<T> trip(G);
    {
      std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
      for (int64_t r = 0; r < q; ++r)
        for (int64_t k = t.nn_rowptr[r]; k < t.nn_rowptr[r + 1]; ++k) {
          if (t.nn_val[k] == 0.0) continue;
          const int32_t leaf = t.point_index[t.nn_col[k]];
          trip[pos[leaf]++] = T{r, t.nn_col[k], t.nn_val[k]};
        }
    }
    // one entry per distinct fine point of a bucket; entries numbered leaf by
    // leaf, so each leaf fills its own slice of the arrays
    std::vector<int64_t> ecnt(N + 1, 0);
#pragma omp parallel for schedule(dynamic, 256) if (G > 65536)
    for (int32_t i = 0; i < N; ++i) {
      int64_t c = 0;
      for (int64_t k = cnt[i]; k < cnt[i + 1]; ++k) c += (k == cnt[i] || trip[k].q != trip[k - 1].q);
      ecnt[i + 1] = c;
    }
    for (int32_t i = 0; i < N; ++i) ecnt[i + 1] += ecnt[i];
    const int64_t E = ecnt[N];
    t.src_pos.resize(3 * E);
    t.src_origin.resize(E);
    t.src_goff.resize(E + 1);
    t.src_gidx.resize(G);
    t.src_gw.resize(G);
#pragma omp parallel for schedule(dynamic, 256) if (G > 65536)
    for (int32_t i = 0; i < N; ++i) {
      t.src_start[i] = ecnt[i];
      int64_t e = ecnt[i];
      for (int64_t k = cnt[i]; k < cnt[i + 1]; ++k) {
        const T& x = trip[k];
        if (k == cnt[i] || x.q != trip[k - 1].q) {
          t.src_goff[e] = k;
          std::memcpy(&t.src_pos[3 * e], &t.fine[3 * x.q], 3 * sizeof(double));
          t.src_origin[e] = x.q;
          ++e;
        }
        t.src_gidx[k] = (int32_t)t.pot_rank[x.col];
        t.src_gw[k] = x.w;
      }
    }
    t.src_goff[E] = G;
    t.src_start[N] = E;
  }
  return NNK_OK;
}

// ------------------------------------------------------------------ NN --
void nearest_matrix(const double* coarse, int64_t n, const double* fine, int64_t q,
                    std::vector<int64_t>& rowptr, std::vector<int32_t>& col,
                    std::vector<double>& val) {
  rowptr.assign(q + 1, 0);
  col.clear();
  val.clear();
  if (n == 0 || q == 0) return;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = coarse[d];
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], coarse[3 * i + d]);
      hi[d] = std::max(hi[d], coarse[3 * i + d]);
    }
  double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
  if (!(ext > 0)) ext = 1.0;
  // about two coarse points per occupied cell for surface-like sets
  int g = (int)std::ceil(std::cbrt((double)n / 2.0));
  g = std::max(1, std::min(g, 512));
  const double h = ext / g * (1.0 + 1e-12);
  int dim[3];
  for (int d = 0; d < 3; ++d) dim[d] = std::max(1, std::min(g, (int)std::floor((hi[d] - lo[d]) / h) + 1));
  auto cell_of = [&](const double* p, int* c) {
    for (int d = 0; d < 3; ++d) {
      long v = (long)std::floor((p[d] - lo[d]) / h);
      c[d] = (int)std::max(0L, std::min((long)dim[d] - 1, v));
    }
  };
  const int64_t ncell = (int64_t)dim[0] * dim[1] * dim[2];
  std::vector<int64_t> cstart(ncell + 1, 0), cpts(n);
  std::vector<int64_t> pc(n);
  for (int64_t i = 0; i < n; ++i) {
    int c[3];
    cell_of(coarse + 3 * i, c);
    pc[i] = ((int64_t)c[2] * dim[1] + c[1]) * dim[0] + c[0];
    cstart[pc[i] + 1]++;
  }
  for (int64_t k = 0; k < ncell; ++k) cstart[k + 1] += cstart[k];
  {
    std::vector<int64_t> pos(cstart.begin(), cstart.end() - 1);
    for (int64_t i = 0; i < n; ++i) cpts[pos[pc[i]]++] = i;  // ascending within a cell
  }
  std::vector<std::vector<int32_t>> hits(q);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t r = 0; r < q; ++r) {
    const double* f = fine + 3 * r;
    int c[3];
    cell_of(f, c);
    double best = INFINITY;
    std::vector<int32_t>& hv = hits[r];
    for (int ring = 0;; ++ring) {
      for (int dz = -ring; dz <= ring; ++dz)
        for (int dy = -ring; dy <= ring; ++dy)
          for (int dx = -ring; dx <= ring; ++dx) {
            if (std::max({std::abs(dx), std::abs(dy), std::abs(dz)}) != ring) continue;
            const int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= dim[0] || y >= dim[1] || z >= dim[2]) continue;
            const int64_t cell = ((int64_t)z * dim[1] + y) * dim[0] + x;
            for (int64_t k = cstart[cell]; k < cstart[cell + 1]; ++k) {
              const int64_t j = cpts[k];
              const double ddx = f[0] - coarse[3 * j];
              const double ddy = f[1] - coarse[3 * j + 1];
              const double ddz = f[2] - coarse[3 * j + 2];
              // (dx^2 + dy^2) + dz^2, each operation rounded (no contraction)
              const double d2 = (ddx * ddx + ddy * ddy) + ddz * ddz;
              if (d2 < best) {
                best = d2;
                hv.clear();
                hv.push_back((int32_t)j);
              } else if (d2 == best) {
                hv.push_back((int32_t)j);
              }
            }
          }
      // every unvisited coarse point lies outside the visited block of cells;
      // stop once the block's nearest face is strictly farther than best.
      bool all = (c[0] - ring <= 0 && c[1] - ring <= 0 && c[2] - ring <= 0 &&
                  c[0] + ring >= dim[0] - 1 && c[1] + ring >= dim[1] - 1 && c[2] + ring >= dim[2] - 1);
      if (all) break;
      double dmin = INFINITY;
      for (int d = 0; d < 3; ++d) {
        if (c[d] - ring > 0) dmin = std::min(dmin, f[d] - (lo[d] + (c[d] - ring) * h));
        if (c[d] + ring < dim[d] - 1) dmin = std::min(dmin, (lo[d] + (c[d] + ring + 1) * h) - f[d]);
      }
      if (dmin > 0 && best < dmin * dmin * (1.0 - 1e-9)) break;
    }
    std::sort(hv.begin(), hv.end());
  }
  for (int64_t r = 0; r < q; ++r) rowptr[r + 1] = rowptr[r] + (int64_t)hits[r].size();
  col.resize(rowptr[q]);
  val.resize(rowptr[q]);
  for (int64_t r = 0; r < q; ++r) {
    const double w = 1.0 / (double)hits[r].size();
    for (size_t k = 0; k < hits[r].size(); ++k) {
      col[rowptr[r] + k] = hits[r][k];
      val[rowptr[r] + k] = w;
    }
  }
}

void merge_forest(const std::vector<const HostTree*>& trees, HostTree& f) {
  f = HostTree();
  if (trees.empty()) throw Error(NNK_E_ARG, "empty forest");
  f.params = trees[0]->params;
  auto cat_csr = [](Csr& dst, const Csr& src, int32_t node_off, bool first) {
    const int64_t base = dst.off.empty() ? 0 : dst.off.back();
    if (first) dst.off.push_back(0);
    for (size_t r = 1; r < src.off.size(); ++r) dst.off.push_back(base + src.off[r]);
    for (int32_t v : src.idx) dst.idx.push_back(v + node_off);
  };
  int64_t E = 0, G = 0, T = 0, npot = 0, ntgt = 0;
  for (size_t k = 0; k < trees.size(); ++k) {
    const HostTree& t = *trees[k];
    if (t.params.nearest != f.params.nearest) throw Error(NNK_E_ARG, "forest trees must agree on NEAREST");
    const int32_t off = f.nodes;
    f.roots.push_back(off);
    f.max_level = std::max(f.max_level, t.max_level);
    for (int32_t n = 0; n < t.nodes; ++n) {
      f.level.push_back(t.level[n]);
      f.parent.push_back(t.parent[n] < 0 ? -1 : t.parent[n] + off);
      f.child0.push_back(t.child0[n] < 0 ? -1 : t.child0[n] + off);
      f.ix.push_back(t.ix[n]);
      f.iy.push_back(t.iy[n]);
      f.iz.push_back(t.iz[n]);
      f.tleaf.push_back(t.tleaf[n]);
      f.pleaf.push_back(t.pleaf[n]);
      f.group.push_back((int32_t)k);
    }
    f.corners.insert(f.corners.end(), t.corners.begin(), t.corners.end());
    cat_csr(f.U, t.U, off, k == 0);
    cat_csr(f.V, t.V, off, k == 0);
    cat_csr(f.W, t.W, off, k == 0);
    cat_csr(f.X, t.X, off, k == 0);
    if (k == 0) {
      f.src_start.push_back(0);
      f.tgt_start.push_back(0);
      f.src_goff.push_back(0);
    }
    for (int32_t n = 0; n < t.nodes; ++n) {
      f.src_start.push_back(E + t.src_start[n + 1]);
      f.tgt_start.push_back(T + t.tgt_start[n + 1]);
    }
    f.src_pos.insert(f.src_pos.end(), t.src_pos.begin(), t.src_pos.end());
    for (size_t e = 1; e < t.src_goff.size(); ++e) f.src_goff.push_back(G + t.src_goff[e]);
    for (int32_t r : t.src_gidx) f.src_gidx.push_back((int32_t)(r + npot));
    for (int64_t o : t.src_origin) f.src_origin.push_back(o + (t.params.nearest ? f.q : npot));
    f.src_gw.insert(f.src_gw.end(), t.src_gw.begin(), t.src_gw.end());
    for (int32_t r : t.tgt_row) f.tgt_row.push_back((int32_t)(r + ntgt));
    f.tgt_pos.insert(f.tgt_pos.end(), t.tgt_pos.begin(), t.tgt_pos.end());
    f.nodes += t.nodes;
    E += t.src_start[t.nodes];
    G += t.src_goff.empty() ? 0 : t.src_goff.back();
    T += (int64_t)t.tgt_row.size();
    npot += t.n_pot;
    ntgt += t.n_tgt;
    f.n += t.n;
    f.q += t.q;
  }
  if (npot > INT32_MAX || ntgt > INT32_MAX) throw Error(NNK_E_ARG, "forest too large for 32-bit rows");
  f.n_pot = npot;
  f.n_tgt = ntgt;
  f.by_level.assign(f.max_level + 1, {});
  for (int32_t n = 0; n < f.nodes; ++n) f.by_level[f.level[n]].push_back(n);
}

void nearest_reference_weights(int64_t q, const int64_t* rowptr, const int32_t* col, double* val,
                               double block_size) {
  if (q <= 0) return;
  const double bn = std::floor(block_size * 134217728.0 / (9.0 * (double)q));  // nearestMatrix.m:23
  if (!(bn >= 1.0))
    throw Error(NNK_E_ARG, "blockSize too small: nearestMatrix.m builds no block (blockNodes = 0)");
  const int64_t block = bn > (double)q ? q : (int64_t)bn;
  std::vector<int64_t> cm;
  std::vector<double> w;
  for (int64_t s = 0; s < q; s += block) {
    const int64_t e = std::min(q, s + block);
    const int64_t a = rowptr[s], b = rowptr[e];
    // the tie weights 1/k_q in row-major order (by fine point, then coarse index)
    w.clear();
    for (int64_t r = s; r < e; ++r) {
      for (int64_t k = rowptr[r] + 1; k < rowptr[r + 1]; ++k)
        if (col[k] <= col[k - 1]) throw Error(NNK_E_ARG, "NN columns must ascend within a row");
      for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k) w.push_back(1.0 / (double)(rowptr[r + 1] - rowptr[r]));
    }
    // the tied pairs in column-major order (by coarse index, then fine point)
    cm.resize(b - a);
    for (int64_t k = a; k < b; ++k) cm[k - a] = k;
    std::stable_sort(cm.begin(), cm.end(), [&](int64_t x, int64_t y) { return col[x] < col[y]; });
    for (size_t j = 0; j < cm.size(); ++j) val[cm[j]] = w[j];
  }
}

}  // namespace nnk
