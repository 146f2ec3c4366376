// GPU construction of the octree's node structure and of the nearest-
// neighbour matrix, bit-identical to the host builders in tree.cpp.
//
// Octree (Classes/OcTree.m:155-222): the tree is grown level by level.  The
// work proportional to the points -- the octant of every point of a node that
// divides and the stable partition of the node's range by octant -- runs on
// the GPU in fixed-size chunks of a node's range: a count pass, prefix sums
// over the chunks of each node (host, O(nodes)), and a scatter pass that
// ranks each point among its chunk's points of the same octant in index
// order.  Midpoints, the strict `p > centre` test and the per-level node
// bookkeeping follow the host builder exactly; the reference's depth-first
// block numbering is assigned at the end from the divided nodes' preorder
// ranks: the children of the r-th divided node (preorder, root r = 0) are
// ids 1 + 8 r + k.
//
// nearestMatrix (Tools/Nearest/nearestMatrix.m:17-41): one thread per fine
// point searches rings of grid cells around it with the host's grid, the
// squared distance formed as (dx^2 + dy^2) + dz^2 in round-to-nearest FP64
// with no fused multiply-add, so exact ties (weight 1/k) match the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "common.h"
#include "tree.h"

namespace nnk {

namespace {

constexpr int kChunk = 2048;  // points per chunk (256 threads x 8)
constexpr int kMaxTies = 16;  // nearest coarse points kept per fine point on the device

struct ChunkT {
  int start;   // first position in `order`
  int len;
  int node;    // dividing node of the level (index into ctr)
  int pad;
};

__device__ __forceinline__ int octant(const double* __restrict__ pts, int p, const double* c) {
  const double* x = pts + 3 * (long long)p;
  return 4 * (x[0] > c[0]) + 2 * (x[1] > c[1]) + (x[2] > c[2]);
}

// counts[chunk][8]
__global__ void tree_count_kernel(const double* __restrict__ pts, const int* __restrict__ order,
                                  const ChunkT* __restrict__ chunks, const double* __restrict__ ctr,
                                  int* __restrict__ counts) {
  const ChunkT ch = chunks[blockIdx.x];
  const double c[3] = {ctr[3 * ch.node], ctr[3 * ch.node + 1], ctr[3 * ch.node + 2]};
  __shared__ int sc[8];
  if (threadIdx.x < 8) sc[threadIdx.x] = 0;
  __syncthreads();
  int loc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = threadIdx.x; k < ch.len; k += blockDim.x) loc[octant(pts, order[ch.start + k], c)]++;
  for (int o = 0; o < 8; ++o)
    if (loc[o]) atomicAdd(&sc[o], loc[o]);
  __syncthreads();
  if (threadIdx.x < 8) counts[8 * blockIdx.x + threadIdx.x] = sc[threadIdx.x];
}

// Stable scatter: thread t handles points [8t, 8t+8) of the chunk; its rank
// among the chunk's points of octant o is the exclusive prefix over threads
// of their counts of o plus the rank inside its own 8 points.
__global__ void __launch_bounds__(256) tree_scatter_kernel(const double* __restrict__ pts,
                                                           const int* __restrict__ order,
                                                           const ChunkT* __restrict__ chunks,
                                                           const double* __restrict__ ctr,
                                                           const int* __restrict__ base, int* __restrict__ out) {
  const ChunkT ch = chunks[blockIdx.x];
  const double c[3] = {ctr[3 * ch.node], ctr[3 * ch.node + 1], ctr[3 * ch.node + 2]};
  __shared__ int pre[8][257];
  const int t = threadIdx.x;
  int oc[8], pv[8];
  int loc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int k = 8 * t + i;
    oc[i] = -1;
    if (k < ch.len) {
      pv[i] = order[ch.start + k];
      oc[i] = octant(pts, pv[i], c);
      loc[oc[i]]++;
    }
  }
#pragma unroll
  for (int o = 0; o < 8; ++o) pre[o][t + 1] = loc[o];
  if (t == 0)
    for (int o = 0; o < 8; ++o) pre[o][0] = 0;
  __syncthreads();
  if (t < 8) {  // exclusive prefix of octant t over the 256 threads (serial, 256 adds)
    int s = 0;
    for (int k = 0; k <= 256; ++k) {
      const int v = pre[t][k];
      pre[t][k] = s;
      s += v;
    }
  }
  __syncthreads();
  int run[8];
#pragma unroll
  for (int o = 0; o < 8; ++o) run[o] = pre[o][t + 1];
#pragma unroll
  for (int i = 0; i < 8; ++i)
    if (oc[i] >= 0) out[base[8 * blockIdx.x + oc[i]] + run[oc[i]]++] = pv[i];
}

// ---------------------------------------------------------- nearest matrix
struct Grid {
  double lo[3];
  double h;
  int dim[3];
};

__device__ __forceinline__ void cell_of(const Grid& g, const double* p, int* c) {
  for (int d = 0; d < 3; ++d) {
    const long long v = (long long)floor((p[d] - g.lo[d]) / g.h);
    c[d] = (int)max(0LL, min((long long)g.dim[d] - 1, v));
  }
}

// Per fine point: the nearest coarse points (ascending, up to kMaxTies; the
// count is exact and larger counts are redone on the host).
__global__ void nn_search_kernel(Grid g, const double* __restrict__ coarse, const long long* __restrict__ cstart,
                                 const int* __restrict__ cpts, const double* __restrict__ fine, long long q,
                                 int* __restrict__ nhit, int* __restrict__ hits) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= q) return;
  const double f[3] = {fine[3 * r], fine[3 * r + 1], fine[3 * r + 2]};
  int c[3];
  cell_of(g, f, c);
  double best = INFINITY;
  int cnt = 0;
  int hv[kMaxTies];
  auto visit = [&](int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= g.dim[0] || y >= g.dim[1] || z >= g.dim[2]) return;
    const long long cell = ((long long)z * g.dim[1] + y) * g.dim[0] + x;
    for (long long k = cstart[cell]; k < cstart[cell + 1]; ++k) {
      const int j = cpts[k];
      const double ddx = __dsub_rn(f[0], coarse[3LL * j]);
      const double ddy = __dsub_rn(f[1], coarse[3LL * j + 1]);
      const double ddz = __dsub_rn(f[2], coarse[3LL * j + 2]);
      const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
      if (d2 < best) {
        best = d2;
        cnt = 0;
      }
      if (d2 == best) {
        // keep the smallest column indices, ascending
        if (cnt < kMaxTies) {
          int pos = cnt;
          while (pos > 0 && hv[pos - 1] > j) {
            hv[pos] = hv[pos - 1];
            --pos;
          }
          hv[pos] = j;
        } else if (hv[kMaxTies - 1] > j) {
          int pos = kMaxTies - 1;
          while (pos > 0 && hv[pos - 1] > j) {
            hv[pos] = hv[pos - 1];
            --pos;
          }
          hv[pos] = j;
        }
        ++cnt;
      }
    }
  };
  for (int ring = 0;; ++ring) {
    // the cells at Chebyshev distance `ring` from c, shell only
    for (int dz = -ring; dz <= ring; ++dz) {
      if (c[2] + dz < 0 || c[2] + dz >= g.dim[2]) continue;
      for (int dy = -ring; dy <= ring; ++dy) {
        if (c[1] + dy < 0 || c[1] + dy >= g.dim[1]) continue;
        if (abs(dz) == ring || abs(dy) == ring) {
          for (int dx = -ring; dx <= ring; ++dx) visit(c[0] + dx, c[1] + dy, c[2] + dz);
        } else {
          visit(c[0] - ring, c[1] + dy, c[2] + dz);
          if (ring > 0) visit(c[0] + ring, c[1] + dy, c[2] + dz);
        }
      }
    }
    const bool all = (c[0] - ring <= 0 && c[1] - ring <= 0 && c[2] - ring <= 0 && c[0] + ring >= g.dim[0] - 1 &&
                      c[1] + ring >= g.dim[1] - 1 && c[2] + ring >= g.dim[2] - 1);
    if (all) break;
    double dmin = INFINITY;
    for (int d = 0; d < 3; ++d) {
      if (c[d] - ring > 0) dmin = fmin(dmin, f[d] - (g.lo[d] + (c[d] - ring) * g.h));
      if (c[d] + ring < g.dim[d] - 1) dmin = fmin(dmin, (g.lo[d] + (c[d] + ring + 1) * g.h) - f[d]);
    }
    if (dmin > 0 && best < dmin * dmin * (1.0 - 1e-9)) break;
  }
  nhit[r] = cnt;
  for (int k = 0; k < min(cnt, kMaxTies); ++k) hits[r * kMaxTies + k] = hv[k];
}

}  // namespace

void nearest_matrix_gpu(nnk_ctx* ctx, const double* coarse, int64_t n, const double* fine, int64_t q,
                        std::vector<int64_t>& rowptr, std::vector<int32_t>& col, std::vector<double>& val) {
  rowptr.assign(q + 1, 0);
  col.clear();
  val.clear();
  if (n == 0 || q == 0) return;
  if (n > INT32_MAX) throw Error(NNK_E_ARG, "too many coarse points for 32-bit columns");
  // the host builder's grid (tree.cpp, nearest_matrix)
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = coarse[d];
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], coarse[3 * i + d]);
      hi[d] = std::max(hi[d], coarse[3 * i + d]);
    }
  double ext = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
  if (!(ext > 0)) ext = 1.0;
  int gn = (int)std::ceil(std::cbrt((double)n / 2.0));
  gn = std::max(1, std::min(gn, 512));
  Grid g;
  g.h = ext / gn * (1.0 + 1e-12);
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = lo[d];
    g.dim[d] = std::max(1, std::min(gn, (int)std::floor((hi[d] - lo[d]) / g.h) + 1));
  }
  auto cell_host = [&](const double* p) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      long v = (long)std::floor((p[d] - lo[d]) / g.h);
      c[d] = (int)std::max(0L, std::min((long)g.dim[d] - 1, v));
    }
    return ((int64_t)c[2] * g.dim[1] + c[1]) * g.dim[0] + c[0];
  };
  const int64_t ncell = (int64_t)g.dim[0] * g.dim[1] * g.dim[2];
  std::vector<long long> cstart(ncell + 1, 0);
  std::vector<int> cpts(n);
  std::vector<int64_t> pc(n);
  for (int64_t i = 0; i < n; ++i) {
    pc[i] = cell_host(coarse + 3 * i);
    cstart[pc[i] + 1]++;
  }
  for (int64_t k = 0; k < ncell; ++k) cstart[k + 1] += cstart[k];
  {
    std::vector<long long> pos(cstart.begin(), cstart.end() - 1);
    for (int64_t i = 0; i < n; ++i) cpts[pos[pc[i]]++] = (int)i;
  }
  cudaStream_t st = ctx->stream;
  DBuf<double> dco, dfi;
  DBuf<long long> dcs;
  DBuf<int> dcp, dnh(q), dh((size_t)q * kMaxTies);
  dco.alloc(3 * n);
  dfi.alloc(3 * q);
  NNK_CUDA(cudaMemcpyAsync(dco.p, coarse, 3 * n * sizeof(double), cudaMemcpyHostToDevice, st));
  NNK_CUDA(cudaMemcpyAsync(dfi.p, fine, 3 * q * sizeof(double), cudaMemcpyHostToDevice, st));
  dcs.upload(cstart, st);
  dcp.upload(cpts, st);
  nn_search_kernel<<<(unsigned)((q + 127) / 128), 128, 0, st>>>(g, dco.p, dcs.p, dcp.p, dfi.p, q, dnh.p, dh.p);
  NNK_CHECK_LAUNCH();
  std::vector<int> nh(q), h((size_t)q * kMaxTies);
  NNK_CUDA(cudaMemcpyAsync(nh.data(), dnh.p, q * sizeof(int), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaMemcpyAsync(h.data(), dh.p, h.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  for (int64_t r = 0; r < q; ++r) rowptr[r + 1] = rowptr[r] + nh[r];
  col.resize(rowptr[q]);
  val.resize(rowptr[q]);
  for (int64_t r = 0; r < q; ++r) {
    const int k = nh[r];
    const double w = 1.0 / (double)k;
    if (k <= kMaxTies) {
      for (int i = 0; i < k; ++i) {
        col[rowptr[r] + i] = h[(size_t)r * kMaxTies + i];
        val[rowptr[r] + i] = w;
      }
    } else {
      // more ties than kept on the device: every coarse point at that
      // distance, by a full host scan of this row
      const double* f = fine + 3 * r;
      double best = INFINITY;
      std::vector<int32_t> hv;
      for (int64_t j = 0; j < n; ++j) {
        const double dx = f[0] - coarse[3 * j], dy = f[1] - coarse[3 * j + 1], dz = f[2] - coarse[3 * j + 2];
        volatile double a = dx * dx, b = dy * dy, cc = dz * dz;
        volatile double ab = a + b;
        const double d2 = ab + cc;
        if (d2 < best) {
          best = d2;
          hv.clear();
        }
        if (d2 == best) hv.push_back((int32_t)j);
      }
      for (int i = 0; i < k; ++i) {
        col[rowptr[r] + i] = hv[i];
        val[rowptr[r] + i] = w;
      }
    }
  }
}

int build_nodes_gpu(nnk_ctx* ctx, HostTree& t, std::string& msg) {
  cudaStream_t st = ctx->stream;
  const int64_t n = t.n;
  if (n > INT32_MAX) throw Error(NNK_E_ARG, "too many points for the GPU tree builder");
  DBuf<double> dpts;
  dpts.upload(t.pts, st);
  std::vector<int> order0(n);
  for (int64_t i = 0; i < n; ++i) order0[i] = (int)i;
  DBuf<int> ord[2];
  ord[0].upload(order0, st);
  ord[1].alloc(n);
  int cur = 0;
  // nodes in creation (breadth-first) order
  struct NodeB {
    int level, parent, child0;  // child0: first child (breadth-first index) or -1
    int ix, iy, iz;
    double c[6];
    int64_t start, count;
  };
  std::vector<NodeB> nb;
  {
    const double* r = &t.corners[0];
    nb.push_back(NodeB{0, -1, -1, 0, 0, 0, {r[0], r[1], r[2], r[3], r[4], r[5]}, 0, n});
  }
  size_t lev_first = 0, lev_end = 1;
  for (int L = 0; lev_end > lev_first; ++L) {
    // OcTree.m:168-170: the depth check runs for every visited node
    if (L + 1 >= t.params.max_depth) {
      msg = "Max level reached: Increase Max Depth";
      return NNK_E_MAXDEPTH;
    }
    std::vector<size_t> div;
    for (size_t i = lev_first; i < lev_end; ++i)
      if (nb[i].count > t.capacity) div.push_back(i);
    if (div.empty()) break;
    // centres (mean([lo;hi],1)) and chunks of the dividing nodes' ranges
    std::vector<double> ctr(3 * div.size());
    std::vector<ChunkT> chunks;
    for (size_t d = 0; d < div.size(); ++d) {
      const NodeB& u = nb[div[d]];
      for (int a = 0; a < 3; ++a) ctr[3 * d + a] = (u.c[a] + u.c[3 + a]) / 2.0;
      for (int64_t s = 0; s < u.count; s += kChunk)
        chunks.push_back(ChunkT{(int)(u.start + s), (int)std::min<int64_t>(kChunk, u.count - s), (int)d, 0});
    }
    DBuf<double> dctr;
    DBuf<ChunkT> dch;
    DBuf<int> dcnt(8 * chunks.size()), dbase(8 * chunks.size());
    dctr.upload(ctr, st);
    dch.upload(chunks, st);
    tree_count_kernel<<<(unsigned)chunks.size(), 256, 0, st>>>(dpts.p, ord[cur].p, dch.p, dctr.p, dcnt.p);
    NNK_CHECK_LAUNCH();
    std::vector<int> cnt(8 * chunks.size()), base(8 * chunks.size());
    NNK_CUDA(cudaMemcpyAsync(cnt.data(), dcnt.p, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    NNK_CUDA(cudaStreamSynchronize(st));
    // per dividing node: octant totals (children's counts) and chunk bases
    std::vector<std::array<int64_t, 8>> tot(div.size());
    for (auto& a : tot) a.fill(0);
    for (size_t k = 0; k < chunks.size(); ++k)
      for (int o = 0; o < 8; ++o) tot[chunks[k].node][o] += cnt[8 * k + o];
    std::vector<std::array<int64_t, 8>> run(div.size());
    for (size_t d = 0; d < div.size(); ++d) {
      int64_t s = nb[div[d]].start;
      for (int o = 0; o < 8; ++o) {
        run[d][o] = s;
        s += tot[d][o];
      }
    }
    for (size_t k = 0; k < chunks.size(); ++k)
      for (int o = 0; o < 8; ++o) {
        base[8 * k + o] = (int)run[chunks[k].node][o];
        run[chunks[k].node][o] += cnt[8 * k + o];
      }
    dbase.upload(base, st);
    NNK_CUDA(cudaMemcpyAsync(ord[1 - cur].p, ord[cur].p, n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    tree_scatter_kernel<<<(unsigned)chunks.size(), 256, 0, st>>>(dpts.p, ord[cur].p, dch.p, dctr.p, dbase.p,
                                                                  ord[1 - cur].p);
    NNK_CHECK_LAUNCH();
    cur = 1 - cur;
    // children of every dividing node, in order (Dividenode, OcTree.m:181-222)
    const size_t next_first = nb.size();
    for (size_t d = 0; d < div.size(); ++d) {
      const size_t u = div[d];
      nb[u].child0 = (int)nb.size();
      int64_t s = nb[u].start;
      const double* lo = nb[u].c;
      const double* hi = nb[u].c + 3;
      const double* cc = &ctr[3 * d];
      for (int o = 0; o < 8; ++o) {
        const int bx = (o >> 2) & 1, by = (o >> 1) & 1, bz = o & 1;
        NodeB ch{L + 1, (int)u, -1, 2 * nb[u].ix + bx, 2 * nb[u].iy + by, 2 * nb[u].iz + bz,
                 {bx ? cc[0] : lo[0], by ? cc[1] : lo[1], bz ? cc[2] : lo[2], bx ? hi[0] : cc[0],
                  by ? hi[1] : cc[1], bz ? hi[2] : cc[2]},
                 s, tot[d][o]};
        nb.push_back(ch);
        s += tot[d][o];
      }
    }
    lev_first = next_first;
    lev_end = nb.size();
  }
  // depth-first block numbering: divided nodes' preorder ranks from the
  // number of divided nodes in each subtree
  const size_t NB = nb.size();
  std::vector<int64_t> ndiv(NB, 0), rank(NB, -1);
  for (size_t i = NB; i-- > 0;) {
    if (nb[i].child0 < 0) continue;
    ndiv[i] = 1;
    for (int k = 0; k < 8; ++k) ndiv[i] += ndiv[nb[i].child0 + k];
  }
  std::vector<int32_t> id(NB, -1);
  id[0] = 0;
  if (nb[0].child0 >= 0) rank[0] = 0;
  for (size_t i = 0; i < NB; ++i) {  // parents precede their children
    if (nb[i].child0 < 0) continue;
    int64_t r = rank[i] + 1;
    for (int k = 0; k < 8; ++k) {
      const int c = nb[i].child0 + k;
      id[c] = (int32_t)(1 + 8 * rank[i] + k);
      if (nb[c].child0 >= 0) {
        rank[c] = r;
        r += ndiv[c];
      }
    }
  }
  t.nodes = (int32_t)NB;
  t.level.assign(NB, 0);
  t.parent.assign(NB, -1);
  t.child0.assign(NB, -1);
  t.ix.assign(NB, 0);
  t.iy.assign(NB, 0);
  t.iz.assign(NB, 0);
  t.corners.assign(6 * NB, 0.0);
  t.pstart.assign(NB, 0);
  t.pcount.assign(NB, 0);
  for (size_t i = 0; i < NB; ++i) {
    const int32_t k = id[i];
    t.level[k] = nb[i].level;
    t.parent[k] = nb[i].parent < 0 ? -1 : id[nb[i].parent];
    t.child0[k] = nb[i].child0 < 0 ? -1 : id[nb[i].child0];
    t.ix[k] = nb[i].ix;
    t.iy[k] = nb[i].iy;
    t.iz[k] = nb[i].iz;
    std::copy(nb[i].c, nb[i].c + 6, &t.corners[6 * (size_t)k]);
    t.pstart[k] = nb[i].start;
    t.pcount[k] = nb[i].count;
  }
  std::vector<int> ordh(n);
  NNK_CUDA(cudaMemcpyAsync(ordh.data(), ord[cur].p, n * sizeof(int), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  t.order.assign(ordh.begin(), ordh.end());
  return NNK_OK;
}

}  // namespace nnk
