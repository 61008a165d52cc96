// chainmesh.cu -- the chain-mesh cell sort on the device.
//
// Reference: chainmesh_create -> sort (src/chainmesh.cpp:139-213) ->
// particles_sort (src/particles.cpp:414-444).  The reference bisects the
// chain box recursively (split dim = the LAST dim with span > 1, mid =
// begin + span/2) and partitions the particle range in place at each node
// with a two-pointer (Hoare) pass on x[dim] >= fixed32(mid * (1.0/C)).
//
// Device design (no recursion, no per-node launches):
//  1. keys:   each particle's chain cell from the reference's own split
//             thresholds thr[m] = fixed32(m * (1.0/C)), so "x < thr[mid]" and
//             "cell < mid" are the same predicate bit for bit;
//  2. counts: per-cell histogram (warp-aggregated atomics) + exclusive scan
//             gives the cell offsets, which the recursion leaves in
//             (z, y, x)-lexicographic order;
//  3. PARITY order: every node of the recursion tree owns a contiguous
//             position range that the offsets already determine, so all nodes
//             of one depth are partitioned together.  A two-pointer pass swaps
//             the i-th misplaced element of the left part (ascending) with the
//             i-th misplaced element of the right part (descending); one
//             depth level is therefore one flag scan, one slot scatter and one
//             pairwise swap over all positions.  Levels = 3 * ceil(log2 C).
//     FAST order: a stable counting sort (input order inside each cell).
//  4. gather: the accumulated permutation is applied once to x, y, z, vx, vy,
//             vz and rung, and positions are packed as int4 for the PP kernel.
#include "tpm_internal.cuh"

#include <algorithm>
#include <cstring>

namespace tpm {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Cell coordinate of raw position r along one axis: the largest m with
// r >= thr[m] (thr[0] = 0).  The integer estimate floor(r*C/2^32) is within
// one of it; the threshold table settles the boundary exactly.
__device__ __forceinline__ int cell_coord(uint32_t r, int C, const uint32_t* __restrict__ thr) {
  int c = (int)(((uint64_t)r * (uint64_t)C) >> 32);
  if (c + 1 < C && r >= __ldg(thr + c + 1)) c++;
  else if (c > 0 && r < __ldg(thr + c)) c--;
  return c;
}

__global__ void k_cell_keys(int64_t n, const uint32_t* __restrict__ x, const uint32_t* __restrict__ y,
                            const uint32_t* __restrict__ z, const uint32_t* __restrict__ thr, int C,
                            uint32_t* __restrict__ key, int32_t* __restrict__ idx,
                            int32_t* __restrict__ count) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = i < n;
  uint32_t k = 0xffffffffu;
  if (live) {
    const int cx = cell_coord(x[i], C, thr);
    const int cy = cell_coord(y[i], C, thr);
    const int cz = cell_coord(z[i], C, thr);
    k = ((uint32_t)cz * (uint32_t)C + (uint32_t)cy) * (uint32_t)C + (uint32_t)cx;
    key[i] = k;
    idx[i] = (int32_t)i;
  }
  // warp-aggregated histogram: one atomic per distinct key in the warp
  const unsigned live_mask = __ballot_sync(0xffffffffu, live);
  if (live) {
    const unsigned peers = __match_any_sync(live_mask, k);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(count + k, __popc(peers));
  }
}

// Block-wide exclusive scan of one int per thread (kScanThreads threads).
__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_tot, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (kScanThreads / 32) ? warp_tot[lane] : 0;
    int wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < (kScanThreads / 32)) warp_tot[lane] = wi - w;
    if (lane == (kScanThreads / 32) - 1) *total = wi;
  }
  __syncthreads();
  const int r = warp_tot[warp] + incl - v;
  return r;
}

// Exclusive scan of in[0..n) into out[0..n], out[n] = total, in ONE block
// (used for per-block sums and cell counts of modest size).
__global__ void __launch_bounds__(kScanThreads) k_scan_single(const int32_t* __restrict__ in, int64_t n,
                                                              int32_t* __restrict__ out) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  int carry = 0;
  for (int64_t base = 0; base < n; base += kScanTile) {
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
      v[k] = i < n ? in[i] : 0;
      s += v[k];
    }
    int off = block_exclusive_scan(s, warp_tot, &total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
      const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
      if (i < n) out[i] = off;
      off += v[k];
    }
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// Multi-block exclusive scan, pass 1: per-block totals.
__global__ void __launch_bounds__(kScanThreads) k_scan_blocksum(const int32_t* __restrict__ in, int64_t n,
                                                                int32_t* __restrict__ bsum) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    s += i < n ? in[i] : 0;
  }
  block_exclusive_scan(s, warp_tot, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// pass 3: block-local exclusive scan plus the scanned block offset.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int32_t* __restrict__ in, int64_t n,
                                                             const int32_t* __restrict__ boff,
                                                             int32_t* __restrict__ out) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  int off = block_exclusive_scan(s, warp_tot, &total) + boff[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = off;
    off += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = boff[gridDim.x];
}

// cellof[p] = the cell whose final range holds position p (one warp per cell).
__global__ void k_cellof(int64_t ncell, const int32_t* __restrict__ begin, int32_t* __restrict__ cellof) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= ncell) return;
  const int32_t b = begin[w], e = begin[w + 1];
  for (int32_t p = b + lane; p < e; p += 32) cellof[p] = (int32_t)w;
}

struct LevelArgs {
  int64_t n;
  int C;
  int level;
  const int32_t* __restrict__ cellof;
  const uint32_t* __restrict__ key;
  const int32_t* __restrict__ begin;
  const TreeNode* __restrict__ tree;
  const int* __restrict__ depth;
};

// The recursion node that owns position p at this depth: its position range
// [b, e), the split point pm (first position of the right child), the split
// dim's mid cell and the particle's coordinate along that dim.  Returns false
// when the cell holding p is already a leaf at this depth.
__device__ __forceinline__ bool node_of(const LevelArgs& a, int64_t p, int32_t& b, int32_t& pm,
                                        int32_t& e, bool& is_left_flag) {
  const int cell = a.cellof[p];
  const int C = a.C;
  const int cx = cell % C, cy = (cell / C) % C, cz = cell / (C * C);
  const int dz = __ldg(a.depth + cz), dy = __ldg(a.depth + cy), dx = __ldg(a.depth + cx);
  const uint32_t k = a.key[p];
  const int kx = (int)(k % (uint32_t)C), ky = (int)((k / (uint32_t)C) % (uint32_t)C),
            kz = (int)(k / ((uint32_t)C * (uint32_t)C));
  int l = a.level;
  const int64_t CC = (int64_t)C * C;
  if (l < dz) {
    const TreeNode t = a.tree[cz * kMaxTreeDepth + l];
    b = __ldg(a.begin + t.lo * CC);
    pm = __ldg(a.begin + t.mid * CC);
    e = __ldg(a.begin + t.hi * CC);
    is_left_flag = kz < t.mid;
    return true;
  }
  l -= dz;
  if (l < dy) {
    const TreeNode t = a.tree[cy * kMaxTreeDepth + l];
    const int64_t base = (int64_t)cz * C;
    b = __ldg(a.begin + (base + t.lo) * C);
    pm = __ldg(a.begin + (base + t.mid) * C);
    e = __ldg(a.begin + (base + t.hi) * C);
    is_left_flag = ky < t.mid;
    return true;
  }
  l -= dy;
  if (l < dx) {
    const TreeNode t = a.tree[cx * kMaxTreeDepth + l];
    const int64_t base = ((int64_t)cz * C + cy) * C;
    b = __ldg(a.begin + base + t.lo);
    pm = __ldg(a.begin + base + t.mid);
    e = __ldg(a.begin + base + t.hi);
    is_left_flag = kx < t.mid;
    return true;
  }
  return false;
}

// f(p) = 1 when the particle at p belongs to the LEFT child (x < xmid).
__device__ __forceinline__ int level_flag(const LevelArgs& a, int64_t p) {
  int32_t b, pm, e;
  bool left;
  if (p >= a.n || !node_of(a, p, b, pm, e, left)) return 0;
  return left ? 1 : 0;
}

__global__ void __launch_bounds__(kScanThreads) k_level_blocksum(LevelArgs a, int32_t* __restrict__ bsum) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) s += level_flag(a, base + (int64_t)threadIdx.x * kScanItems + k);
  block_exclusive_scan(s, warp_tot, &total);
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_level_prefix(LevelArgs a, const int32_t* __restrict__ boff,
                                                               int32_t* __restrict__ prefix) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    v[k] = level_flag(a, base + (int64_t)threadIdx.x * kScanItems + k);
    s += v[k];
  }
  int off = block_exclusive_scan(s, warp_tot, &total) + boff[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    const int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < a.n) prefix[i] = off;
    off += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) prefix[a.n] = boff[gridDim.x];
}

// Right-part elements that belong left (x < xmid) are the two-pointer's
// swap partners, met in descending order: the k-th from the end of the node
// goes to slot[b + k].
__global__ void k_level_slots(LevelArgs a, const int32_t* __restrict__ prefix, int32_t* __restrict__ slot) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  int32_t b, pm, e;
  bool left;
  if (!node_of(a, p, b, pm, e, left)) return;
  if (p >= pm && left) {
    const int32_t k = prefix[e] - prefix[p] - 1;  // flagged elements in (p, e)
    slot[b + k] = (int32_t)p;
  }
}

// Left-part elements that belong right swap with their partner: the k-th
// such element from the start of the node pairs with slot[b + k].
__global__ void k_level_swap(LevelArgs a, const int32_t* __restrict__ prefix, const int32_t* __restrict__ slot,
                             uint32_t* __restrict__ key, int32_t* __restrict__ idx) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  int32_t b, pm, e;
  bool left;
  if (!node_of(a, p, b, pm, e, left)) return;
  if (p < pm && !left) {
    const int32_t k = (int32_t)(p - b) - (prefix[p] - prefix[b]);  // unflagged in [b, p)
    const int32_t q = slot[b + k];
    const uint32_t kp = key[p], kq = key[q];
    const int32_t ip = idx[p], iq = idx[q];
    key[p] = kq;
    key[q] = kp;
    idx[p] = iq;
    idx[q] = ip;
  }
}

// FAST order: stable counting sort.  rank-in-cell of particle i = number of
// earlier particles with the same key; computed by a scatter with atomics
// followed by a per-cell sort of the original indices.
__global__ void k_fast_scatter(int64_t n, const uint32_t* __restrict__ key, const int32_t* __restrict__ begin,
                               int32_t* __restrict__ fill, int32_t* __restrict__ idx_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t k = key[i];
  const int32_t pos = begin[k] + atomicAdd(fill + k, 1);
  idx_out[pos] = (int32_t)i;
}

// One warp per cell: insertion-merge of the cell's original indices into
// ascending order (cells are small; large cells fall back to a shared-memory
// odd-even transposition loop with a bounded trip count).
__global__ void k_fast_cellsort(int64_t ncell, const int32_t* __restrict__ begin, int32_t* __restrict__ idx) {
  const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= ncell) return;
  const int32_t b = begin[w], e = begin[w + 1];
  const int32_t len = e - b;
  // odd-even transposition sort: len phases, each lane handles pairs
  for (int32_t phase = 0; phase < len; phase++) {
    for (int32_t j = b + (phase & 1) + 2 * lane; j + 1 < e; j += 64) {
      const int32_t u = idx[j], v = idx[j + 1];
      if (u > v) {
        idx[j] = v;
        idx[j + 1] = u;
      }
    }
    __syncwarp();
  }
}

__global__ void k_gather(int64_t n, const int32_t* __restrict__ idx, const uint32_t* __restrict__ x,
                         const uint32_t* __restrict__ y, const uint32_t* __restrict__ z,
                         const float* __restrict__ vx, const float* __restrict__ vy,
                         const float* __restrict__ vz, const int8_t* __restrict__ rung,
                         uint32_t* __restrict__ x2, uint32_t* __restrict__ y2, uint32_t* __restrict__ z2,
                         float* __restrict__ vx2, float* __restrict__ vy2, float* __restrict__ vz2,
                         int8_t* __restrict__ rung2, int4* __restrict__ pos4) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t i = idx[p];
  const uint32_t a = x[i], b = y[i], c = z[i];
  x2[p] = a;
  y2[p] = b;
  z2[p] = c;
  vx2[p] = vx[i];
  vy2[p] = vy[i];
  vz2[p] = vz[i];
  rung2[p] = rung[i];
  pos4[p] = make_int4((int)a, (int)b, (int)c, 0);
}

int scan_exclusive(tpm_ctx* c, const int32_t* in, int64_t n, int32_t* out) {
  if (n <= (int64_t)kScanTile * 64) {
    k_scan_single<<<1, kScanThreads, 0, c->stream>>>(in, n, out);
    c->launches++;
  } else {
    const int nb = ceil_div(n, kScanTile);
    k_scan_blocksum<<<nb, kScanThreads, 0, c->stream>>>(in, n, c->blocksum);
    k_scan_single<<<1, kScanThreads, 0, c->stream>>>(c->blocksum, nb, c->blocksum + nb + 1);
    k_scan_apply<<<nb, kScanThreads, 0, c->stream>>>(in, n, c->blocksum + nb + 1, out);
    c->launches += 3;
  }
  TPM_CUDA_TRY(cudaGetLastError());
  return TPM_OK;
}

}  // namespace

// Host tables: split thresholds and the 1-D bisection tree.
int sort_init(tpm_ctx* c) {
  const int C = c->C;
  std::vector<uint32_t> thr(C + 1);
  // mid_x = mid_box * Ninv with Ninv = 1.0 / N; xmid = fixed32(mid_x)
  // (src/chainmesh.cpp:171,198-199; src/particles.cpp:417; tigerpm/fixed.hpp:73-75).
  const double Cinv = 1.0 / C;
  for (int m = 0; m < C; m++) thr[m] = (uint32_t)(4294967296.0 * (m * Cinv));
  thr[C] = 0xffffffffu;
  std::vector<TreeNode> tree((size_t)C * kMaxTreeDepth, TreeNode{0, 0, 0, 0});
  std::vector<int> depth(C);
  int maxd = 0;
  for (int v = 0; v < C; v++) {
    int lo = 0, hi = C, k = 0;
    while (hi - lo > 1) {
      if (k >= kMaxTreeDepth) return fail(TPM_ERR_INVALID, "chain_dim too large");
      const int mid = lo + (hi - lo) / 2;
      tree[(size_t)v * kMaxTreeDepth + k] = TreeNode{lo, mid, hi, 0};
      if (v < mid) hi = mid;
      else lo = mid;
      k++;
    }
    depth[v] = k;
    maxd = std::max(maxd, k);
  }
  c->max_depth1d = maxd;
  TPM_CUDA_TRY(cudaMemcpy(c->thr, thr.data(), sizeof(uint32_t) * (C + 1), cudaMemcpyHostToDevice));
  TPM_CUDA_TRY(cudaMemcpy(c->tree, tree.data(), sizeof(TreeNode) * tree.size(), cudaMemcpyHostToDevice));
  TPM_CUDA_TRY(cudaMemcpy(c->depth1d, depth.data(), sizeof(int) * C, cudaMemcpyHostToDevice));
  return TPM_OK;
}

int chainmesh_sort(tpm_ctx* c) {
  const int64_t n = c->n;
  const int C = c->C;
  const int64_t ncell = (int64_t)C * C * C;
  cudaStream_t s = c->stream;
  stage_begin(c, kStSort);
  TPM_CUDA_TRY(cudaMemsetAsync(c->cell_count, 0, sizeof(int32_t) * (ncell + 1), s));
  if (n > 0) {
    k_cell_keys<<<ceil_div(n, 256), 256, 0, s>>>(n, c->x, c->y, c->z, c->thr, C, c->key, c->idx,
                                                  c->cell_count);
    c->launches++;
  }
  int rc = scan_exclusive(c, c->cell_count, ncell, c->cell_begin);
  if (rc) return rc;
  if (n > 0) {
    if (c->opt.sort_mode == TPM_SORT_FAST) {
      TPM_CUDA_TRY(cudaMemsetAsync(c->cell_count, 0, sizeof(int32_t) * (ncell + 1), s));
      k_fast_scatter<<<ceil_div(n, 256), 256, 0, s>>>(n, c->key, c->cell_begin, c->cell_count, c->prefix);
      k_fast_cellsort<<<ceil_div(ncell * 32, 256), 256, 0, s>>>(ncell, c->cell_begin, c->prefix);
      c->launches += 2;
      TPM_CUDA_TRY(cudaMemcpyAsync(c->idx, c->prefix, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    } else {
      k_cellof<<<ceil_div(ncell * 32, 256), 256, 0, s>>>(ncell, c->cell_begin, c->cellof);
      c->launches++;
      const int nb = ceil_div(n, kScanTile);
      const int levels = 3 * c->max_depth1d;
      for (int l = 0; l < levels; l++) {
        LevelArgs a{n, C, l, c->cellof, c->key, c->cell_begin, c->tree, c->depth1d};
        k_level_blocksum<<<nb, kScanThreads, 0, s>>>(a, c->blocksum);
        k_scan_single<<<1, kScanThreads, 0, s>>>(c->blocksum, nb, c->blocksum + nb + 1);
        k_level_prefix<<<nb, kScanThreads, 0, s>>>(a, c->blocksum + nb + 1, c->prefix);
        k_level_slots<<<ceil_div(n, 256), 256, 0, s>>>(a, c->prefix, c->slot);
        k_level_swap<<<ceil_div(n, 256), 256, 0, s>>>(a, c->prefix, c->slot, c->key, c->idx);
        c->launches += 5;
      }
    }
    k_gather<<<ceil_div(n, 256), 256, 0, s>>>(n, c->idx, c->x, c->y, c->z, c->vx, c->vy, c->vz, c->rung,
                                               c->x2, c->y2, c->z2, c->vx2, c->vy2, c->vz2, c->rung2,
                                               c->pos4);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
    std::swap(c->x, c->x2);
    std::swap(c->y, c->y2);
    std::swap(c->z, c->z2);
    std::swap(c->vx, c->vx2);
    std::swap(c->vy, c->vy2);
    std::swap(c->vz, c->vz2);
    std::swap(c->rung, c->rung2);
  }
  stage_end(c, kStSort);
  c->sorted = true;
  c->host_cells_valid = false;
  return TPM_OK;
}

}  // namespace tpm
