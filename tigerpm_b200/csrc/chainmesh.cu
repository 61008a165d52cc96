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
#ifndef TPM_LEVEL_PER
#define TPM_LEVEL_PER 4
#endif
// consecutive positions per thread in the slot and swap passes (a multiple of 4)
constexpr int kLevelPer = TPM_LEVEL_PER;
static_assert(kLevelPer % 4 == 0, "positions are read four at a time");
static_assert(kScanTile == kScanTileElems, "scan tiles must match the status and block-sum arrays");

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

// The recursion node that owns positions of final cell `cell` at this depth:
// its position range [b, e), the split point pm (first position of the right
// child), the split dim (0..2) and mid cell.  Returns false when the cell is
// already a leaf at this depth.
struct Node {
  int32_t b, pm, e;
  int dim, mid;
  bool live;
};

__device__ __forceinline__ Node node_of_cell(const LevelArgs& a, int cell) {
  Node nd;
  const int C = a.C;
  const int cx = cell % C, cy = (cell / C) % C, cz = cell / (C * C);
  const int dz = __ldg(a.depth + cz), dy = __ldg(a.depth + cy), dx = __ldg(a.depth + cx);
  int l = a.level;
  const int64_t CC = (int64_t)C * C;
  nd.live = true;
  if (l < dz) {
    const TreeNode t = a.tree[cz * kMaxTreeDepth + l];
    nd.b = __ldg(a.begin + t.lo * CC);
    nd.pm = __ldg(a.begin + t.mid * CC);
    nd.e = __ldg(a.begin + t.hi * CC);
    nd.dim = 2;
    nd.mid = t.mid;
    return nd;
  }
  l -= dz;
  if (l < dy) {
    const TreeNode t = a.tree[cy * kMaxTreeDepth + l];
    const int64_t base = (int64_t)cz * C;
    nd.b = __ldg(a.begin + (base + t.lo) * C);
    nd.pm = __ldg(a.begin + (base + t.mid) * C);
    nd.e = __ldg(a.begin + (base + t.hi) * C);
    nd.dim = 1;
    nd.mid = t.mid;
    return nd;
  }
  l -= dy;
  if (l < dx) {
    const TreeNode t = a.tree[cx * kMaxTreeDepth + l];
    const int64_t base = ((int64_t)cz * C + cy) * C;
    nd.b = __ldg(a.begin + base + t.lo);
    nd.pm = __ldg(a.begin + base + t.mid);
    nd.e = __ldg(a.begin + base + t.hi);
    nd.dim = 0;
    nd.mid = t.mid;
    return nd;
  }
  nd.live = false;
  nd.b = nd.pm = nd.e = 0;
  nd.dim = 0;
  nd.mid = 0;
  return nd;
}

// f = 1 when the particle with cell key k belongs to the node's LEFT child
// (its coordinate along the split dim is below mid, i.e. x < xmid).
__device__ __forceinline__ int left_flag(const Node& nd, uint32_t k, int C) {
  if (!nd.live) return 0;
  const uint32_t uc = (uint32_t)C;
  const int c = nd.dim == 0 ? (int)(k % uc) : nd.dim == 1 ? (int)((k / uc) % uc) : (int)(k / (uc * uc));
  return c < nd.mid ? 1 : 0;
}

// Four consecutive int32 entries from position p (a multiple of 4, so the
// 16-byte load is aligned) when all four are below n; else one by one.
__device__ __forceinline__ int4 load4(const int32_t* __restrict__ a, int64_t p, int64_t n) {
  if (p + 4 <= n) return *reinterpret_cast<const int4*>(a + p);
  int4 r = make_int4(0, 0, 0, 0);
  if (p < n) r.x = a[p];
  if (p + 1 < n) r.y = a[p + 1];
  if (p + 2 < n) r.z = a[p + 2];
  return r;
}

// Node lookups are cached while consecutive positions share a final cell
// (cells hold many particles), which removes most dependent loads.
struct NodeCache {
  int cell = -1;
  Node nd;
  __device__ __forceinline__ const Node& get(const LevelArgs& a, int c) {
    if (c != cell) {
      cell = c;
      nd = node_of_cell(a, c);
    }
    return nd;
  }
};

// Decoupled look-back scan status word: stamp (30 bits) | flag (2 bits) | value (32 bits).
constexpr unsigned long long kFlagAgg = 1ull, kFlagIncl = 2ull;
__device__ __forceinline__ unsigned long long pack_status(unsigned stamp, unsigned long long flag, int value) {
  return ((unsigned long long)stamp << 34) | (flag << 32) | (unsigned long long)(unsigned)value;
}

// One partition level, part 1: the left-child flags of every position and
// their exclusive prefix, in a single pass (chained scan with decoupled
// look-back; tiles are taken in launch order through an atomic counter, so
// every predecessor a tile waits on is already running).  The look-back is
// done by one warp, 32 predecessor tiles at a time; its spin is bounded: on
// expiry the tile records kErrTimeout and uses what it has summed.  Cells,
// keys and prefixes move 16 bytes per load / store; four resident blocks per
// SM (32 registers) beat three at 40 registers without the bound.
__global__ void __launch_bounds__(kScanThreads, 4) k_level_scan(LevelArgs a, unsigned stamp, int* __restrict__ counter,
                                                             unsigned long long* __restrict__ status,
                                                             int32_t* __restrict__ prefix, int* __restrict__ err) {
  __shared__ int warp_tot[32];
  __shared__ int total;
  __shared__ int tile_s;
  __shared__ int excl_s;
  if (threadIdx.x == 0) tile_s = atomicAdd(counter, 1);
  __syncthreads();
  const int tile = tile_s;
  const int64_t base = (int64_t)tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
  NodeCache cache;
  static_assert(kScanItems % 4 == 0, "positions are read four at a time");
  // cells and keys of the thread's positions, four at a time (16-byte loads)
#pragma unroll
  for (int k = 0; k < kScanItems; k += 4) {
    const int4 c = load4(a.cellof, base + k, a.n);
    const int4 q = load4(reinterpret_cast<const int32_t*>(a.key), base + k, a.n);
    const int cof[4] = {c.x, c.y, c.z, c.w}, ky[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int64_t p = base + k + i;
      v[k + i] = 0;
      if (p < a.n) v[k + i] = left_flag(cache.get(a, cof[i]), (uint32_t)ky[i], a.C);
      s += v[k + i];
    }
  }
  const int off = block_exclusive_scan(s, warp_tot, &total);
  if (threadIdx.x < 32) {
    // warp-parallel look-back: lane l reads the status of tile (top - l);
    // once all 32 are published, the aggregates up to the closest inclusive
    // prefix are summed, else the window moves 32 tiles back
    const int lane = threadIdx.x;
    const int agg = total;
    int excl = 0;
    if (tile == 0) {
      if (lane == 0) atomicExch(status, pack_status(stamp, kFlagIncl, agg));
    } else {
      if (lane == 0) atomicExch(status + tile, pack_status(stamp, kFlagAgg, agg));
      int top = tile - 1;
      long long spins = 0;
      while (true) {
        const int j = top - lane;
        unsigned long long f = kFlagIncl;  // before tile 0: an inclusive zero
        int v = 0;
        if (j >= 0) {
          const unsigned long long w = *reinterpret_cast<volatile unsigned long long*>(status + j);
          f = (unsigned)(w >> 34) == stamp ? (w >> 32) & 3ull : 0ull;
          v = (int)(unsigned)(w & 0xffffffffull);
        }
        if (__any_sync(0xffffffffu, f == 0)) {
          if (++spins > (1ll << 22)) {
            if (lane == 0) atomicOr(err, kErrTimeout);
            break;
          }
          continue;
        }
        const unsigned incl = __ballot_sync(0xffffffffu, f == kFlagIncl);
        const int first = incl ? __ffs(incl) - 1 : 32;
        int sum = lane <= first ? v : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        excl += sum;
        if (incl) break;
        top -= 32;
      }
      if (lane == 0) atomicExch(status + tile, pack_status(stamp, kFlagIncl, excl + agg));
    }
    if (lane == 0) excl_s = excl;
  }
  __syncthreads();
  int run = excl_s + off;
  int pr[kScanItems];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    pr[k] = run;
    run += v[k];
  }
  if (base + kScanItems <= a.n) {
#pragma unroll
    for (int k = 0; k < kScanItems; k += 4)
      *reinterpret_cast<int4*>(prefix + base + k) = make_int4(pr[k], pr[k + 1], pr[k + 2], pr[k + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
      if (base + k < a.n) prefix[base + k] = pr[k];
  }
  if (base < a.n && base + kScanItems >= a.n) prefix[a.n] = run;  // the thread holding position n-1
}

// Part 2: right-part elements that belong left (x < xmid) are the
// two-pointer's swap partners, met in descending order: the k-th from the
// end of the node goes to slot[b + k].
__global__ void __launch_bounds__(256) k_level_slots(LevelArgs a, const int32_t* __restrict__ prefix,
                                                     int32_t* __restrict__ slot) {
  const int64_t p0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * kLevelPer;
  NodeCache cache;
  int cof[kLevelPer], ky[kLevelPer], pf[kLevelPer];
#pragma unroll
  for (int h = 0; h < kLevelPer; h += 4) {
    const int4 c4 = load4(a.cellof, p0 + h, a.n);
    const int4 k4 = load4(reinterpret_cast<const int32_t*>(a.key), p0 + h, a.n);
    const int4 f4 = load4(prefix, p0 + h, a.n);
    cof[h] = c4.x, cof[h + 1] = c4.y, cof[h + 2] = c4.z, cof[h + 3] = c4.w;
    ky[h] = k4.x, ky[h + 1] = k4.y, ky[h + 2] = k4.z, ky[h + 3] = k4.w;
    pf[h] = f4.x, pf[h + 1] = f4.y, pf[h + 2] = f4.z, pf[h + 3] = f4.w;
  }
#pragma unroll
  for (int k = 0; k < kLevelPer; k++) {
    const int64_t p = p0 + k;
    if (p >= a.n) return;
    const Node& nd = cache.get(a, cof[k]);
    if (!nd.live || p < nd.pm) continue;
    if (left_flag(nd, (uint32_t)ky[k], a.C)) {
      const int32_t kk = prefix[nd.e] - pf[k] - 1;  // flagged elements in (p, e)
      slot[nd.b + kk] = (int32_t)p;
    }
  }
}

// Part 3: left-part elements that belong right swap with their partner: the
// k-th such element from the start of the node pairs with slot[b + k].
__global__ void __launch_bounds__(256) k_level_swap(LevelArgs a, const int32_t* __restrict__ prefix,
                                                    const int32_t* __restrict__ slot, uint32_t* __restrict__ key,
                                                    int32_t* __restrict__ idx) {
  const int64_t p0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) * kLevelPer;
  NodeCache cache;
  // cells and prefixes are read-only here; keys are swapped by other
  // threads (at right-part positions), so they are read one by one
  int cof[kLevelPer], pf[kLevelPer];
#pragma unroll
  for (int h = 0; h < kLevelPer; h += 4) {
    const int4 c4 = load4(a.cellof, p0 + h, a.n);
    const int4 f4 = load4(prefix, p0 + h, a.n);
    cof[h] = c4.x, cof[h + 1] = c4.y, cof[h + 2] = c4.z, cof[h + 3] = c4.w;
    pf[h] = f4.x, pf[h + 1] = f4.y, pf[h + 2] = f4.z, pf[h + 3] = f4.w;
  }
#pragma unroll
  for (int k = 0; k < kLevelPer; k++) {
    const int64_t p = p0 + k;
    if (p >= a.n) return;
    const Node& nd = cache.get(a, cof[k]);
    if (!nd.live || p >= nd.pm) continue;
    if (!left_flag(nd, key[p], a.C)) {
      const int32_t kk = (int32_t)(p - nd.b) - (pf[k] - prefix[nd.b]);  // unflagged in [b, p)
      const int32_t q = slot[nd.b + kk];
      const uint32_t kp = key[p], kq = key[q];
      const int32_t ip = idx[p], iq = idx[q];
      key[p] = kq;
      key[q] = kp;
      idx[p] = iq;
      idx[q] = ip;
    }
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

// The sorted set back into the current arrays (batch members keep fixed
// device addresses across steps).
__global__ void k_copy_back(int64_t n, const uint32_t* __restrict__ x2, const uint32_t* __restrict__ y2,
                            const uint32_t* __restrict__ z2, const float* __restrict__ vx2,
                            const float* __restrict__ vy2, const float* __restrict__ vz2,
                            const int8_t* __restrict__ rung2, uint32_t* __restrict__ x, uint32_t* __restrict__ y,
                            uint32_t* __restrict__ z, float* __restrict__ vx, float* __restrict__ vy,
                            float* __restrict__ vz, int8_t* __restrict__ rung) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  x[p] = x2[p];
  y[p] = y2[p];
  z[p] = z2[p];
  vx[p] = vx2[p];
  vy[p] = vy2[p];
  vz[p] = vz2[p];
  rung[p] = rung2[p];
}

// One block for up to four tiles; above that, block sums + one-block scan of
// them + apply (three launches of a few microseconds each against 0.22 ms
// for one block walking the 262,144 cells of a 64^3 chain mesh).
int scan_exclusive(tpm_ctx* c, const int32_t* in, int64_t n, int32_t* out) {
  if (n <= (int64_t)kScanTile * 4) {
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
      // per-level tile counters (zeroed once) and look-back status words
      int* counters = c->cell_count;  // reused: C^3 + 1 >= levels ints after the scan above
      unsigned long long* status = c->scan_status;
      TPM_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(int) * (levels + 1), s));
      const int nq = ceil_div(n, kLevelPer);
      for (int l = 0; l < levels; l++) {
        LevelArgs a{n, C, l, c->cellof, c->key, c->cell_begin, c->tree, c->depth1d};
        const unsigned stamp = (unsigned)(++c->scan_stamp & 0x3fffffff);
        k_level_scan<<<nb, kScanThreads, 0, s>>>(a, stamp, counters + l, status, c->prefix, c->d_err);
        k_level_slots<<<ceil_div(nq, 256), 256, 0, s>>>(a, c->prefix, c->slot);
        k_level_swap<<<ceil_div(nq, 256), 256, 0, s>>>(a, c->prefix, c->slot, c->key, c->idx);
        c->launches += 3;
      }
    }
    k_gather<<<ceil_div(n, 256), 256, 0, s>>>(n, c->idx, c->x, c->y, c->z, c->vx, c->vy, c->vz, c->rung,
                                               c->x2, c->y2, c->z2, c->vx2, c->vy2, c->vz2, c->rung2,
                                               c->pos4);
    c->launches++;
    TPM_CUDA_TRY(cudaGetLastError());
    if (c->stable_buffers) {
      k_copy_back<<<ceil_div(n, 256), 256, 0, s>>>(n, c->x2, c->y2, c->z2, c->vx2, c->vy2, c->vz2, c->rung2, c->x,
                                                   c->y, c->z, c->vx, c->vy, c->vz, c->rung);
      c->launches++;
      TPM_CUDA_TRY(cudaGetLastError());
    } else {
      std::swap(c->x, c->x2);
      std::swap(c->y, c->y2);
      std::swap(c->z, c->z2);
      std::swap(c->vx, c->vx2);
      std::swap(c->vy, c->vy2);
      std::swap(c->vz, c->vz2);
      std::swap(c->rung, c->rung2);
    }
  }
  stage_end(c, kStSort);
  c->sorted = true;
  c->pot_valid = false;  // forces and potentials are not permuted with the particles
  c->host_cells_valid = false;
  return TPM_OK;
}

}  // namespace tpm
