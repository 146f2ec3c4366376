// U/V/W/X interaction lists on the GPU (Classes/OcTree.m:265-366), the
// same arrays as the host builder in tree.cpp (build_lists), bit for bit.
//
// Colleagues (same-level touching nodes, the node itself included) are found
// level by level from the parent's colleagues' children; the `full` flags
// (no empty-potential leaf below) bottom-up.  Then one thread per node
// builds its lists in two passes -- count, then fill at the prefix-sum
// offsets -- and a segmented radix sort orders every node's segment:
//   V (OcTree.m:330-339): children of the parent's non-leaf colleagues other
//     than the parent that do not touch the node;
//   U (:323-327, target leaves): every non-empty potential leaf touching the
//     node, from the ancestors' colleagues and below the node's colleagues;
//   W (:343-361, target leaves): below the node's non-leaf colleagues, the
//     nodes that do not touch it and hold no empty-potential leaf (a complete
//     sibling block merges into its parent), sorted, except that the last
//     merged node (lowest level, then largest id) goes to the end, as the
//     reference's repeated [setdiff(W, children); node] leaves it.
// X (:279-288) is the inverse of W ordered by (position of the node inside
// W(j), then j): a radix sort of (node, position, j) keys.
#include <cub/cub.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "common.h"
#include "tree.h"

namespace nnk {

namespace {

constexpr int kMaxColleagues = 27;
constexpr int kStack = 256;  // DFS stack per thread; 8 + 7 per level of descent is enough below 23 levels

struct ListArgs {
  int N;
  const double* corners;
  const int* level;
  const int* parent;
  const int* child0;
  const unsigned char* pleaf;
  const unsigned char* tleaf;
  const unsigned char* full;
  const int* coll;    // N x 27
  const int* ncoll;   // N
};

__device__ __forceinline__ bool touch(const double* __restrict__ cr, int a, int b) {
  const double* c1 = cr + 6 * (long long)a;
  const double* c2 = cr + 6 * (long long)b;
  return !(c2[0] > c1[3] || c2[3] < c1[0] || c2[1] > c1[4] || c2[4] < c1[1] || c2[2] > c1[5] || c2[5] < c1[2]);
}

// colleagues of the nodes of one level from their parents' colleagues
__global__ void colleagues_kernel(int n, const int* __restrict__ nodes, ListArgs a, int* __restrict__ coll,
                                  int* __restrict__ ncoll) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int c = nodes[j];
  const int P = a.parent[c];
  int cnt = 0;
  int* out = coll + (long long)kMaxColleagues * c;
  for (int q = 0; q < a.ncoll[P]; ++q) {
    const int C = a.coll[(long long)kMaxColleagues * P + q];
    const int c0 = a.child0[C];
    if (c0 < 0) continue;
    for (int k = 0; k < 8; ++k)
      if (touch(a.corners, c, c0 + k) && cnt < kMaxColleagues) out[cnt++] = c0 + k;
  }
  for (int x = 1; x < cnt; ++x) {  // ascending
    const int v = out[x];
    int y = x;
    while (y > 0 && out[y - 1] > v) {
      out[y] = out[y - 1];
      --y;
    }
    out[y] = v;
  }
  ncoll[c] = cnt;
}

__global__ void full_kernel(int n, const int* __restrict__ nodes, const int* __restrict__ child0,
                            const unsigned char* __restrict__ pleaf, unsigned char* __restrict__ full) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int c = nodes[j];
  const int c0 = child0[c];
  if (c0 < 0) {
    full[c] = pleaf[c];
    return;
  }
  unsigned char f = 1;
  for (int k = 0; k < 8; ++k) f &= full[c0 + k];
  full[c] = f;
}

// FILL = false: counts per node (cntU, cntV, cntW); true: the lists at the
// offsets, unsorted, and per node the W entry that goes last (lastW, -1
// none).  err: a DFS stack that would overflow (not expected).
template <bool FILL>
__global__ void lists_kernel(ListArgs a, long long* __restrict__ cntU, long long* __restrict__ cntV,
                             long long* __restrict__ cntW, const long long* __restrict__ offU,
                             const long long* __restrict__ offV, const long long* __restrict__ offW,
                             int* __restrict__ U, int* __restrict__ V, int* __restrict__ W,
                             int* __restrict__ lastW, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  // V
  long long nv = 0;
  if (i > 0) {
    const int P = a.parent[i];
    int* out = FILL ? V + offV[i] : nullptr;
    for (int q = 0; q < a.ncoll[P]; ++q) {
      const int C = a.coll[(long long)kMaxColleagues * P + q];
      const int c0 = a.child0[C];
      if (C == P || c0 < 0) continue;
      for (int k = 0; k < 8; ++k)
        if (!touch(a.corners, c0 + k, i)) {
          if (FILL) out[nv] = c0 + k;
          ++nv;
        }
    }
  }
  if (!FILL) cntV[i] = nv;
  long long nu = 0, nw = 0;
  if (i > 0 && a.tleaf[i]) {
    int stk[kStack];
    // U: the ancestors' leaf colleagues, then the leaves below the node's
    // non-leaf colleagues, each when it is a non-empty potential leaf that
    // touches the node
    int* uo = FILL ? U + offU[i] : nullptr;
    for (int x = i; x >= 0; x = a.parent[x])
      for (int q = 0; q < a.ncoll[x]; ++q) {
        const int C = a.coll[(long long)kMaxColleagues * x + q];
        if (a.child0[C] < 0 && a.pleaf[C] && touch(a.corners, C, i)) {
          if (FILL) uo[nu] = C;
          ++nu;
        }
      }
    for (int q = 0; q < a.ncoll[i]; ++q) {
      const int C = a.coll[(long long)kMaxColleagues * i + q];
      const int c0 = a.child0[C];
      if (c0 < 0) continue;
      int sp = 0;
      for (int k = 0; k < 8; ++k) stk[sp++] = c0 + k;
      while (sp > 0) {
        const int n = stk[--sp];
        if (!touch(a.corners, n, i)) continue;
        const int n0 = a.child0[n];
        if (n0 < 0) {
          if (a.pleaf[n]) {
            if (FILL) uo[nu] = n;
            ++nu;
          }
        } else if (sp + 8 <= kStack) {
          for (int k = 0; k < 8; ++k) stk[sp++] = n0 + k;
        } else {
          atomicOr(err, 1);
        }
      }
    }
    // W
    int* wo = FILL ? W + offW[i] : nullptr;
    int last = -1;
    for (int q = 0; q < a.ncoll[i]; ++q) {
      const int C = a.coll[(long long)kMaxColleagues * i + q];
      const int c0 = a.child0[C];
      if (c0 < 0) continue;
      int sp = 0;
      for (int k = 0; k < 8; ++k) stk[sp++] = c0 + k;
      while (sp > 0) {
        const int n = stk[--sp];
        const int n0 = a.child0[n];
        if (!touch(a.corners, n, i) && a.full[n]) {
          if (FILL) wo[nw] = n;
          ++nw;
          if (n0 >= 0 && (last < 0 || a.level[n] < a.level[last] || (a.level[n] == a.level[last] && n > last)))
            last = n;
          continue;
        }
        if (n0 >= 0) {
          if (sp + 8 <= kStack) {
            for (int k = 0; k < 8; ++k) stk[sp++] = n0 + k;
          } else {
            atomicOr(err, 1);
          }
        }
      }
    }
    if (FILL) lastW[i] = last;
  } else if (FILL) {
    lastW[i] = -1;
  }
  if (!FILL) {
    cntU[i] = nu;
    cntW[i] = nw;
  }
}

// The last merged node of a sorted W segment moves to its end.
__global__ void move_last_kernel(int N, const long long* __restrict__ offW, const int* __restrict__ lastW,
                                 int* __restrict__ W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || lastW[i] < 0) return;
  const long long a = offW[i], b = offW[i + 1];
  const int last = lastW[i];
  long long lo = a, hi = b;  // first position >= last (it is present)
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (W[mid] < last) lo = mid + 1;
    else hi = mid;
  }
  for (long long p = lo; p + 1 < b; ++p) W[p] = W[p + 1];
  if (b > a) W[b - 1] = last;
}

// every node's segment of ids ascending (out of place, then swapped in)
void sort_segments(DBuf<int>& ids, const DBuf<long long>& off, int N, long long total, cudaStream_t st) {
  if (total <= 1) return;
  DBuf<int> out((size_t)total);
  size_t tmp = 0;
  NNK_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp, ids.p, out.p, (int)total, N, off.p, off.p + 1, st));
  DBuf<unsigned char> t(std::max<size_t>(tmp, 1));
  NNK_CUDA(cub::DeviceSegmentedSort::SortKeys(t.p, tmp, ids.p, out.p, (int)total, N, off.p, off.p + 1, st));
  NNK_CUDA(cudaStreamSynchronize(st));  // the temporary storage goes out of scope
  ids = std::move(out);
}

// X keys: (node << 40) | (position in W(j) << 24) | j for every W entry
__global__ void x_keys_kernel(int N, const long long* __restrict__ offW, const int* __restrict__ W,
                              unsigned long long* __restrict__ keys, long long* __restrict__ cntX,
                              int* __restrict__ err) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  if (offW[j + 1] - offW[j] > 65536) atomicOr(err, 2);  // positions need 16 bits
  for (long long k = offW[j]; k < offW[j + 1]; ++k) {
    const unsigned long long node = (unsigned long long)W[k];
    keys[k] = (node << 40) | ((unsigned long long)(k - offW[j]) << 24) | (unsigned long long)j;
    atomicAdd((unsigned long long*)&cntX[W[k]], 1ULL);
  }
}

__global__ void x_ids_kernel(long long n, const unsigned long long* __restrict__ keys, int* __restrict__ X) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) X[k] = (int)(keys[k] & 0xFFFFFFULL);
}

// exclusive prefix sum of n counts into n + 1 offsets (device)
void scan(const long long* cnt, long long* off, int n, cudaStream_t st) {
  NNK_CUDA(cudaMemsetAsync(off, 0, sizeof(long long), st));
  size_t tmp = 0;
  NNK_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, cnt, off + 1, n, st));
  DBuf<unsigned char> t(std::max<size_t>(tmp, 1));
  NNK_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, cnt, off + 1, n, st));
}

template <typename T>
std::vector<T> download(const DBuf<T>& d, size_t n, cudaStream_t st) {
  std::vector<T> h(n);
  if (n) NNK_CUDA(cudaMemcpyAsync(h.data(), d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
  return h;
}

}  // namespace

void build_lists_gpu(nnk_ctx* ctx, HostTree& t) {
  const int N = t.nodes;
  if ((int64_t)N >= (1LL << 24)) throw Error(NNK_E_ARG, "too many nodes for the GPU list builder");
  cudaStream_t st = ctx->stream;
  DBuf<double> cr;
  DBuf<int> lev, par, ch0, coll, ncoll, lvl;
  DBuf<unsigned char> pl, tl, full;
  cr.upload(t.corners, st);
  lev.upload(t.level, st);
  par.upload(t.parent, st);
  ch0.upload(t.child0, st);
  pl.upload(t.pleaf, st);
  tl.upload(t.tleaf, st);
  full.alloc(N);
  coll.alloc((size_t)kMaxColleagues * N);
  ncoll.alloc(N);
  std::vector<int> ln;
  std::vector<int64_t> loff(t.max_level + 2, 0);
  for (int L = 0; L <= t.max_level; ++L) {
    loff[L] = (int64_t)ln.size();
    ln.insert(ln.end(), t.by_level[L].begin(), t.by_level[L].end());
  }
  loff[t.max_level + 1] = (int64_t)ln.size();
  lvl.upload(ln, st);
  {
    const int one = 1, zero = 0;
    NNK_CUDA(cudaMemcpyAsync(ncoll.p, &one, sizeof(int), cudaMemcpyHostToDevice, st));
    NNK_CUDA(cudaMemcpyAsync(coll.p, &zero, sizeof(int), cudaMemcpyHostToDevice, st));
    NNK_CUDA(cudaStreamSynchronize(st));  // the two host words above are on the stack
  }
  ListArgs a{N, cr.p, lev.p, par.p, ch0.p, pl.p, tl.p, full.p, coll.p, ncoll.p};
  for (int L = 1; L <= t.max_level; ++L) {
    const int n = (int)(loff[L + 1] - loff[L]);
    if (n == 0) continue;
    colleagues_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, lvl.p + loff[L], a, coll.p, ncoll.p);
    NNK_CHECK_LAUNCH();
  }
  for (int L = t.max_level; L >= 0; --L) {
    const int n = (int)(loff[L + 1] - loff[L]);
    if (n == 0) continue;
    full_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, lvl.p + loff[L], ch0.p, pl.p, full.p);
    NNK_CHECK_LAUNCH();
  }
  DBuf<long long> cU(N), cV(N), cW(N), oU(N + 1), oV(N + 1), oW(N + 1);
  DBuf<int> err(1);
  err.zero(st);
  const unsigned nb = (unsigned)((N + 127) / 128);
  lists_kernel<false><<<nb, 128, 0, st>>>(a, cU.p, cV.p, cW.p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                          nullptr, err.p);
  NNK_CHECK_LAUNCH();
  scan(cU.p, oU.p, N, st);
  scan(cV.p, oV.p, N, st);
  scan(cW.p, oW.p, N, st);
  long long tot[3];
  NNK_CUDA(cudaMemcpyAsync(&tot[0], oU.p + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaMemcpyAsync(&tot[1], oV.p + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaMemcpyAsync(&tot[2], oW.p + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  NNK_CUDA(cudaStreamSynchronize(st));
  DBuf<int> U(std::max<long long>(tot[0], 1)), V(std::max<long long>(tot[1], 1)), W(std::max<long long>(tot[2], 1));
  DBuf<int> lastW(N);
  lists_kernel<true><<<nb, 128, 0, st>>>(a, nullptr, nullptr, nullptr, oU.p, oV.p, oW.p, U.p, V.p, W.p, lastW.p,
                                         err.p);
  NNK_CHECK_LAUNCH();
  sort_segments(U, oU, N, tot[0], st);
  sort_segments(V, oV, N, tot[1], st);
  sort_segments(W, oW, N, tot[2], st);
  move_last_kernel<<<nb, 128, 0, st>>>(N, oW.p, lastW.p, W.p);
  NNK_CHECK_LAUNCH();
  // X: the inverse of W, by (node, position in W(j), j)
  DBuf<unsigned long long> keys(std::max<long long>(tot[2], 1)), sorted(std::max<long long>(tot[2], 1));
  DBuf<long long> cX(N), oX(N + 1);
  cX.zero(st);
  x_keys_kernel<<<nb, 128, 0, st>>>(N, oW.p, W.p, keys.p, cX.p, err.p);
  NNK_CHECK_LAUNCH();
  DBuf<int> X(std::max<long long>(tot[2], 1));
  if (tot[2] > 0) {
    size_t tmp = 0;
    NNK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp, keys.p, sorted.p, (int)tot[2], 0, 64, st));
    DBuf<unsigned char> tbuf(std::max<size_t>(tmp, 1));
    NNK_CUDA(cub::DeviceRadixSort::SortKeys(tbuf.p, tmp, keys.p, sorted.p, (int)tot[2], 0, 64, st));
    x_ids_kernel<<<(unsigned)((tot[2] + 255) / 256), 256, 0, st>>>(tot[2], sorted.p, X.p);
    NNK_CHECK_LAUNCH();
  }
  scan(cX.p, oX.p, N, st);
  int herr = 0;
  NNK_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  auto csr = [&](const DBuf<long long>& off, const DBuf<int>& ids, long long total, Csr& out) {
    std::vector<long long> o = download(off, (size_t)N + 1, st);
    out.off.assign(o.begin(), o.end());
    out.idx = download(ids, (size_t)total, st);
  };
  csr(oU, U, tot[0], t.U);
  csr(oV, V, tot[1], t.V);
  csr(oW, W, tot[2], t.W);
  csr(oX, X, tot[2], t.X);
  NNK_CUDA(cudaStreamSynchronize(st));
  if (herr & 1) throw Error(NNK_E_STATE, "GPU list builder: DFS stack too small");
  if (herr & 2) throw Error(NNK_E_STATE, "GPU list builder: a W list above 65536 entries");
}

}  // namespace nnk
