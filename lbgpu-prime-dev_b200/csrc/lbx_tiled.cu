// lbx_tiled.cu -- temporal blocking of small 2D lattices.
//
// A 256 x 256 D2Q9 lattice holds 65k nodes: one step is ~0.3 us of work
// spread over 148 SMs, and a step launch (or a graph node) costs more than
// that.  Here one cooperative launch advances the lattice by many steps.
// The lattice is cut into tiles kTX nodes wide and at most kTYMax high;
// per round a block loads its tile with a halo of K nodes into shared
// memory, advances it K steps there (the region still valid shrinks by one
// node per side per step), and writes the tile's own fluid nodes back.
// Rounds alternate between the population array and a scratch copy of it,
// so a round never reads what a slower block of the same round writes.
// The rounds of one launch are even in number: the state ends in the
// population array.
//
// Tile plan.  Where the columns divide the lattice and every tile gets a
// block of its own, each column of tiles is cut into heights that give its
// tiles about equal work per round (fluid node updates, halo included):
// the slowest tile sets the pace, and the fluid fraction of fixed tiles of
// a porous lattice spreads from below 0.3 to near 1.  Between rounds a
// block then waits only for the tiles its halo reads (their round counters,
// polled by one lane each; the wait is bounded in time and records a
// timeout in a status word the host reads at lbx_sync); a counter at r + 1
// also means that tile has finished reading the buffer round r + 1 writes.
// Such a block keeps its tile's nodes in shared memory from round to round
// (they are valid after K steps), reloads only the halo, and stores only
// the strip other halos read (every node it owns in the last round).
// Otherwise the tiles are a fixed grid (the last column may overhang the
// lattice and wrap onto it), blocks may own several, and rounds meet at a
// grid barrier.
//
// In terms of the post-collision populations g the AA pair is one rule
// applied twice: after an even step f[a][n] = g_a(n); a step gathers
// d_a = g_a(n - c_a), or g_opp(a)(n) where n - c_a is solid (the
// half-way bounce-back of the odd step's pull and of the even step's read
// of the slot the odd step's push filled), applies the fused Zou-He / zero
// gradient rows, and collides.  So K steps from the state after an even
// step (K even) end in the state after an even step, in the same slots, and
// the per-node arithmetic is the step kernels' own (collide, face_north,
// face_south): FP64 results are bit-identical to the per-step path.
//
// Eligible: 2D, one substance, no Walsh run, no plane record, faces absent
// or fused, a run of AA pairs whose launch arguments do not change (what
// the graph replay needs too).
#include "lbx.h"
#include "lbx_internal.h"
#include "lbx_kernels.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

namespace cg = cooperative_groups;
using namespace lbx;

namespace {

constexpr int kTX = 32;                // tile width
constexpr int kTYMax = 16;             // tile height, at most
constexpr int kTiledThreads = 512;
constexpr int kMaxNb = 32;             // tiles one halo may read (one warp polls them)
constexpr long long kWaitLimit = 1LL << 20;   // polls of one counter (about a second)

// Steps per round: FP64 six (a halo six nodes deep), FP32 ten (its nodes
// take half the shared memory); measured best of 4/6 and 6/8/10.
template <typename T>
constexpr int tiled_k() { return sizeof(T) == 8 ? 6 : 10; }

// A tile's node lists (tile-local node indices of fluid nodes, row order),
// by the node's distance e from the edge of the tile's region:
//   kListAll    every fluid node (the first load)
//   kListHalo   e < K: the halo, reloaded every round
//   kListStrip  K <= e < 2K: the tile's nodes other halos read
//   kListStep + s (s = 1..K)  e >= s: the nodes step s of a round updates;
//               s = K: the tile's own nodes
constexpr int kListAll = 0, kListHalo = 1, kListStrip = 2, kListStep = 2;

template <int K>
__host__ __device__ constexpr int tiled_region() { return (kTX + 2 * K) * (kTYMax + 2 * K); }

template <typename T, int K>
constexpr size_t tiled_smem()
{
  constexpr int R = tiled_region<K>();
  return 2 * 9 * R * sizeof(T) + R * sizeof(int) + (4 + K) * R * sizeof(unsigned short);
}

// A region node's flags word: bit a (a < 9) the node upstream in direction
// a (n - c_a) is solid; kWSolid the node itself is solid; kWNorth / kWSouth
// its class bits.
constexpr unsigned kWSolid = 1u << 15, kWNorth = 1u << 9, kWSouth = 1u << 10;

// Exclusive prefix sum of one flag per thread over the block; *total gets
// the sum.  `warp_sums` holds kTiledThreads / 32 ints.
__device__ __forceinline__ int block_scan(bool flag, int* warp_sums, int* total)
{
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned ball = __ballot_sync(0xffffffffu, flag);
  const int in_warp = __popc(ball & ((1u << lane) - 1u));
  if (lane == 0) warp_sums[warp] = __popc(ball);
  __syncthreads();
  int before = 0, all = 0;
  for (int w = 0; w < kTiledThreads / 32; ++w) {
    const int c = warp_sums[w];
    if (w < (int)warp) before += c;
    all += c;
  }
  __syncthreads();
  *total = all;
  return before + in_warp;
}

// Round counters: tile t has stored the strips of round r when
// flags[t] >= base + r + 1 (base grows from launch to launch).
__device__ __forceinline__ void publish(int* flag, int value)
{
  __threadfence();
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(flag), "r"(value) : "memory");
}

__device__ __forceinline__ int observe(const int* flag)
{
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
  return v;
}

// f0: the population array (dense [Q][N] or compact [Q][P]); f1: scratch
// of the same shape; fidx: dense -> compact (null for the dense layout).
// plan[t] = (x, y, height) of tile t; nbrs[t][0..kMaxNb): the tiles its
// halo reads, -1 after the last (local waits only).
// Step s of a round updates the fluid nodes at distance >= s from the
// region's edge, from a row-ordered list, so a warp's shared-memory accesses
// are runs of neighbouring nodes and no lane holds a solid node.
template <typename T, int MODEL, int K, bool UNIT_DEN>
__global__ void __launch_bounds__(kTiledThreads, 1)
aa_tiled(StepArgs<T> A, const int* __restrict__ fidx, T* f0, T* f1, long long P, int rounds,
         const int4* __restrict__ plan, int ntiles, const int* __restrict__ nbrs,
         int local_waits, int* flags, int base, int* status)
{
  constexpr int RX = kTX + 2 * K, R = tiled_region<K>();
  constexpr int NL = 3 + K;
  static_assert(R < 65536, "tile list entries are 16-bit");
  extern __shared__ __align__(16) unsigned char smem[];
  T* const b0 = reinterpret_cast<T*>(smem);            // [9][R]
  T* const b1 = b0 + 9 * R;                             // [9][R]
  int* const gidx = reinterpret_cast<int*>(b1 + 9 * R); // [R]: slot of the node, -1 solid
  unsigned short* const lists = reinterpret_cast<unsigned short*>(gidx + R);  // [NL][R]
  unsigned short* const wrd = lists + NL * R;                                // [R] flags words
  __shared__ int warp_sums[kTiledThreads / 32];
  __shared__ int lcount[NL];
  __shared__ int gave_up;
  cg::grid_group grid = cg::this_grid();
  const int LX = A.LX, LY = A.LY;
  const bool keep = ntiles <= (int)gridDim.x;          // one tile per block
  const bool shifted = MODEL != PLAIN_COMP;
  bool tables = false;
  int4 g = keep ? plan[blockIdx.x] : make_int4(0, 0, 0, 0);

  for (int r = 0; r < rounds; ++r) {
    const T* const src = (r & 1) ? f1 : f0;
    T* const dst = (r & 1) ? f0 : f1;
    if (local_waits && r > 0) {
      // this block's tile is blockIdx.x; lane q of warp 0 waits for the q-th
      // tile its halo reads to finish round r - 1
      if (threadIdx.x < 32) {
        int late = 0;
        const int nb = nbrs[blockIdx.x * kMaxNb + threadIdx.x];
        if (nb >= 0) {
          long long polls = 0;
          // every poll is an L2 round trip: no sleep between polls
          while (observe(flags + nb) < base + r) {
            if (++polls >= kWaitLimit || *(volatile int*)status != 0) { late = 1; break; }
          }
        }
        late = __any_sync(0xffffffffu, late);
        if (threadIdx.x == 0) {
          if (late) atomicExch(status, 1);
          gave_up = late;
        }
      }
      __syncthreads();
      if (gave_up) return;          // every thread of the block leaves together
    }
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      if (!keep) g = plan[tile];
      const int x0 = g.x - K, y0 = g.y - K, RY = g.z + 2 * K, RR = RX * RY;
      __syncthreads();                                  // the last tile's stores read smem
      if (!(keep && tables)) {
        for (int i = threadIdx.x; i < RR; i += kTiledThreads) {
          int gx = (x0 + i % RX) % LX, gy = (y0 + i / RX) % LY;
          if (gx < 0) gx += LX;
          if (gy < 0) gy += LY;
          const int n = gx + LX * gy;
          const uint8_t c = A.cls[n];
          wrd[i] = (unsigned short)(((c & CLS_SOLID) ? kWSolid : 0u) | ((c & CLS_NORTH) ? kWNorth : 0u) |
                                    ((c & CLS_SOUTH) ? kWSouth : 0u));
          gidx[i] = (c & CLS_SOLID) ? -1 : (fidx ? fidx[n] : n);
        }
        __syncthreads();
        // upstream solid bits of the nodes a step can update (e >= 1)
        for (int i = threadIdx.x; i < RR; i += kTiledThreads) {
          const int lx = i % RX, ly = i / RX;
          if (lx < 1 || lx > RX - 2 || ly < 1 || ly > RY - 2 || (wrd[i] & kWSolid)) continue;
          unsigned bits = 0;
#pragma unroll
          for (int a = 0; a < 9; ++a)
            if (wrd[i - (cx(a) + RX * cy(a))] & kWSolid) bits |= 1u << a;
          wrd[i] |= (unsigned short)bits;
        }
        __syncthreads();
        for (int l = 0; l < NL; ++l) {
          int cnt = 0;
          for (int c0 = 0; c0 < RR; c0 += kTiledThreads) {
            const int i = c0 + threadIdx.x;
            bool flag = false;
            if (i < RR && !(wrd[i] & kWSolid)) {
              const int lx = i % RX, ly = i / RX;
              const int e = min(min(lx, RX - 1 - lx), min(ly, RY - 1 - ly));
              flag = l == kListAll || (l == kListHalo && e < K) ||
                     (l == kListStrip && e >= K && e < 2 * K) ||
                     (l > kListStep && e >= l - kListStep);
            }
            int tot;
            const int pos = block_scan(flag, warp_sums, &tot);
            if (flag) lists[l * R + cnt + pos] = (unsigned short)i;
            cnt += tot;
          }
          if (threadIdx.x == 0) lcount[l] = cnt;
        }
        __syncthreads();
      }
      {
        const int l = (keep && tables) ? kListHalo : kListAll;
        const unsigned short* const L = lists + l * R;
        const int cnt = lcount[l];
        for (int q = threadIdx.x; q < cnt; q += kTiledThreads) {
          const int i = L[q];
          const int m = gidx[i];
#pragma unroll
          for (int a = 0; a < 9; ++a) b0[a * R + i] = __ldcg(src + a * P + m);
        }
      }
      tables = true;
      __syncthreads();
      T* cur = b0;
      T* nxt = b1;
#pragma unroll 1
      for (int s = 1; s <= K; ++s) {
        const unsigned short* const L = lists + (kListStep + s) * R;
        const int cnt = lcount[kListStep + s];
        for (int q = threadIdx.x; q < cnt; q += kTiledThreads) {
          const int node = L[q];
          const unsigned w = wrd[node];
          T d[9];
#pragma unroll
          for (int a = 0; a < 9; ++a) {
            const int up = node - (cx(a) + RX * cy(a));
            d[a] = ((w >> a) & 1u) ? cur[opp(a) * R + node] : cur[a * R + up];
          }
          if (w & (kWNorth | kWSouth)) {
            if (w & kWNorth)
              face_north<T>(A.face_n[0], A.rho_n[0], A.sc[0].rhoA, A.drho_n[0], shifted, d);
            if (w & kWSouth)
              face_south<T>(A.face_s[0], A.rho_s[0], A.sc[0].rhoA, A.drho_s[0], shifted, d);
          }
          T u[3];
          collide<T, 9, MODEL, false, UNIT_DEN>(A, 0, false, 1, d, u, 0);
#pragma unroll
          for (int a = 0; a < 9; ++a) nxt[a * R + node] = d[a];
        }
        __syncthreads();
        T* const x = cur; cur = nxt; nxt = x;
      }
      // K is even: the round's result is in b0 (cur)
      {
        const bool all = !keep || !local_waits || r + 1 == rounds;
        const int l = all ? kListStep + K : kListStrip;
        const unsigned short* const L = lists + l * R;
        const int cnt = lcount[l];
        for (int q = threadIdx.x; q < cnt; q += kTiledThreads) {
          const int node = L[q];
          if (x0 + node % RX >= LX || y0 + node / RX >= LY) continue;   // overhanging tiles
          const int m = gidx[node];
#pragma unroll
          for (int a = 0; a < 9; ++a) dst[a * P + m] = cur[a * R + node];
        }
      }
    }
    if (r + 1 < rounds) {
      if (local_waits) {
        __syncthreads();                                // the block's stores are issued
        if (threadIdx.x == 0) publish(flags + blockIdx.x, base + r + 1);
      } else {
        grid.sync();
      }
    }
  }
}

// ---- the tile plan (host) ---------------------------------------------------

// Fluid counts over rectangles of the periodic lattice, halos included.
struct FluidSums {
  int LX, LY, ext;
  std::vector<int> s;   // prefix sums over [-ext, LY + ext) x [-ext, LX + ext)

  FluidSums(const std::vector<uint8_t>& solids, int lx, int ly, int e)
      : LX(lx), LY(ly), ext(e), s((size_t)(ly + 2 * e + 1) * (lx + 2 * e + 1), 0)
  {
    const int W = LX + 2 * ext + 1;
    for (int y = 0; y < LY + 2 * ext; ++y)
      for (int x = 0; x < LX + 2 * ext; ++x) {
        const int gx = ((x - ext) % LX + LX) % LX, gy = ((y - ext) % LY + LY) % LY;
        const int f = solids[(size_t)gx + (size_t)LX * gy] != 1;
        s[(size_t)(y + 1) * W + x + 1] = f + s[(size_t)y * W + x + 1] + s[(size_t)(y + 1) * W + x] -
                                         s[(size_t)y * W + x];
      }
  }
  // fluid nodes in [x0, x1) x [y0, y1), -ext <= x0 <= x1 <= LX + ext (same for y)
  int rect(int x0, int y0, int x1, int y1) const
  {
    const int W = LX + 2 * ext + 1;
    x0 += ext; x1 += ext; y0 += ext; y1 += ext;
    return s[(size_t)y1 * W + x1] - s[(size_t)y0 * W + x1] - s[(size_t)y1 * W + x0] +
           s[(size_t)y0 * W + x0];
  }
  // node updates of one round of a tile (x0, y0, h): steps 1..K
  long long work(int x0, int y0, int h, int K) const
  {
    long long w = 0;
    for (int st = 1; st <= K; ++st)
      w += rect(x0 - K + st, y0 - K + st, x0 + kTX + K - st, y0 + h + K - st);
    return w;
  }
};

struct TilePlan {
  std::vector<int4> tiles;
  std::vector<int> nbrs;   // [tiles][kMaxNb]
  bool local = false;
};

// Equal-work columns (see the file comment); false when they do not apply.
bool equal_work_plan(const std::vector<uint8_t>& solids, int LX, int LY, int K, int blocks,
                     TilePlan& out)
{
  if (LX % kTX != 0) return false;
  const int cols = LX / kTX;
  if ((long long)cols * ((LY + kTYMax - 1) / kTYMax) > blocks) return false;
  const FluidSums fs(solids, LX, LY, K + kTYMax);
  auto cut = [&](long long W, std::vector<int4>* tiles) {
    long long n = 0;
    for (int c = 0; c < cols; ++c) {
      for (int y = 0; y < LY;) {
        int h = 1;
        while (h < kTYMax && y + h < LY && fs.work(c * kTX, y, h + 1, K) <= W) ++h;
        if (tiles) tiles->push_back(make_int4(c * kTX, y, h, 0));
        y += h;
        ++n;
      }
    }
    return n;
  };
  long long lo = 0, hi = 0;
  for (int c = 0; c < cols; ++c)
    for (int y = 0; y < LY; y += kTYMax)
      hi = std::max(hi, fs.work(c * kTX, y, std::min(kTYMax, LY - y), K));
  while (lo < hi) {               // the least work bound that needs at most `blocks` tiles
    const long long mid = (lo + hi) / 2;
    if (cut(mid, nullptr) <= blocks) hi = mid; else lo = mid + 1;
  }
  out.tiles.clear();
  cut(lo, &out.tiles);
  // the tiles each halo reads
  std::vector<int> owner((size_t)LX * LY);
  for (size_t t = 0; t < out.tiles.size(); ++t) {
    const int4 g = out.tiles[t];
    for (int y = g.y; y < g.y + g.z; ++y)
      for (int x = g.x; x < g.x + kTX; ++x) owner[(size_t)x + (size_t)LX * y] = (int)t;
  }
  out.nbrs.assign(out.tiles.size() * kMaxNb, -1);
  for (size_t t = 0; t < out.tiles.size(); ++t) {
    const int4 g = out.tiles[t];
    int k = 0;
    int* const row = &out.nbrs[t * kMaxNb];
    for (int y = g.y - K; y < g.y + g.z + K; ++y)
      for (int x = g.x - K; x < g.x + kTX + K; ++x) {
        const int o = owner[(size_t)((x % LX + LX) % LX) + (size_t)LX * ((y % LY + LY) % LY)];
        if (std::find(row, row + k, o) != row + k) continue;
        if (k == kMaxNb) return false;
        row[k++] = o;
      }
  }
  out.local = true;
  return true;
}

TilePlan fixed_plan(int LX, int LY)
{
  TilePlan p;
  for (int y = 0; y < LY; y += kTYMax)
    for (int x = 0; x < LX; x += kTX)
      p.tiles.push_back(make_int4(x, y, std::min(kTYMax, LY - y), 0));
  p.nbrs.assign(p.tiles.size() * kMaxNb, -1);
  return p;
}

lbx_status make_plan(lbx_domain* d, int K)
{
  std::vector<uint8_t> solids((size_t)d->N);
  cudaError_t e = cudaMemcpy(solids.data(), d->solids, (size_t)d->N, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return lbx_internal_fail(LBX_ERR_CUDA, cudaGetErrorString(e));
  TilePlan p;
  if (!equal_work_plan(solids, d->p.LX, d->p.LY, K, d->tiled_grid, p))
    p = fixed_plan(d->p.LX, d->p.LY);
  const int nt = (int)p.tiles.size();
  e = cudaMalloc(&d->tiled_plan, (size_t)nt * sizeof(int4));
  if (e == cudaSuccess) e = cudaMalloc(&d->tiled_nbrs, p.nbrs.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d->tiled_flags, (size_t)(nt + 1) * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(d->tiled_plan, p.tiles.data(), (size_t)nt * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d->tiled_nbrs, p.nbrs.data(), p.nbrs.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d->tiled_flags, 0, (size_t)(nt + 1) * sizeof(int));
  if (e != cudaSuccess) {
    lbx_internal_tiled_free(d);
    return lbx_internal_fail(e == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,
                             cudaGetErrorString(e));
  }
  d->tiled_ntiles = nt;
  d->tiled_local = p.local;
  d->tiled_base = 0;
  return LBX_OK;
}

template <typename T, int MODEL, bool UNIT_DEN>
lbx_status launch(lbx_domain* d, const StepArgs<T>& A, int rounds)
{
  constexpr int K = tiled_k<T>();
  static_assert(K % 2 == 0, "a round must end after an even step");
  constexpr size_t smem = tiled_smem<T, K>();
  const void* fn = (const void*)aa_tiled<T, MODEL, K, UNIT_DEN>;
  if (d->tiled_grid == 0) {
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kTiledThreads, smem);
    if (e != cudaSuccess || !coop || per_sm < 1) {
      cudaGetLastError();
      d->tiled_grid = -1;
    } else {
      d->tiled_grid = sms * per_sm;
    }
  }
  if (d->tiled_grid < 0) return lbx_internal_fail(LBX_ERR_CUDA, "tiled run unavailable on this device");
  const bool compact = d->layout == LBX_LAYOUT_COMPACT;
  const long long P = compact ? d->P : d->N;
  if (!d->tiled_scratch) {
    cudaError_t e = cudaMalloc(&d->tiled_scratch, (size_t)9 * P * sizeof(T));
    if (e != cudaSuccess)
      return lbx_internal_fail(e == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,
                               "tiled scratch allocation failed");
  }
  if (!d->tiled_plan)
    if (lbx_status st = make_plan(d, K)) return st;
  const int ntiles = d->tiled_ntiles;
  if (d->tiled_base + rounds + 1 >= (1 << 30)) {
    // restart the counters before they could wrap
    cudaError_t e = cudaMemsetAsync(d->tiled_flags, 0, (size_t)ntiles * sizeof(int), d->stream);
    if (e != cudaSuccess) return lbx_internal_fail(LBX_ERR_CUDA, cudaGetErrorString(e));
    d->tiled_base = 0;
  }
  StepArgs<T> a = A;
  const int* fidx = compact ? d->fidx : nullptr;
  T* f0 = (T*)(compact ? d->fc : d->f);
  T* f1 = (T*)d->tiled_scratch;
  long long pp = P;
  const int4* plan = d->tiled_plan;
  int nt = ntiles;
  const int* nbrs = d->tiled_nbrs;
  int local = d->tiled_local ? 1 : 0;
  int* flags = d->tiled_flags;
  int* status = d->tiled_flags + ntiles;
  int base = d->tiled_base;
  void* args[] = {&a, &fidx, &f0, &f1, &pp, &rounds, &plan, &nt, &nbrs, &local, &flags, &base, &status};
  const int grid = std::min(d->tiled_grid, ntiles);
  cudaError_t e = cudaLaunchCooperativeKernel(fn, grid, kTiledThreads, args, smem, d->stream);
  if (e != cudaSuccess)
    return lbx_internal_fail(LBX_ERR_CUDA, cudaGetErrorString(e));
  d->tiled_base += rounds;
  d->launches++;
  return LBX_OK;
}

}  // namespace

int lbx_internal_tiled_steps_per_round(const lbx_domain* d)
{
  return d->real_size == 8 ? tiled_k<double>() : tiled_k<float>();
}

template <typename T>
lbx_status lbx_internal_tiled_run(lbx_domain* d, const StepArgs<T>& A, int rounds)
{
  if (rounds <= 0) return LBX_OK;
  if (rounds % 2) return lbx_internal_fail(LBX_ERR_INVALID, "tiled rounds must be even");
  if (d->p.accurate == 0) return launch<T, PLAIN_COMP, false>(d, A, rounds);
  if (d->p.compressible) return launch<T, SHIFTED_COMP, false>(d, A, rounds);
  if (A.sc[0].rhoA == T(1)) return launch<T, SHIFTED_INC, true>(d, A, rounds);
  return launch<T, SHIFTED_INC, false>(d, A, rounds);
}

template lbx_status lbx_internal_tiled_run<float>(lbx_domain*, const StepArgs<float>&, int);
template lbx_status lbx_internal_tiled_run<double>(lbx_domain*, const StepArgs<double>&, int);

void lbx_internal_tiled_free(lbx_domain* d)
{
  cudaFree(d->tiled_scratch);
  cudaFree(d->tiled_flags);
  cudaFree(d->tiled_plan);
  cudaFree(d->tiled_nbrs);
  d->tiled_scratch = nullptr;
  d->tiled_flags = nullptr;
  d->tiled_plan = nullptr;
  d->tiled_nbrs = nullptr;
}

lbx_status lbx_internal_tiled_status(lbx_domain* d)
{
  if (!d->tiled_flags) return LBX_OK;
  const int ntiles = d->tiled_ntiles;
  int st = 0;
  cudaError_t e = cudaMemcpy(&st, d->tiled_flags + ntiles, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return lbx_internal_fail(LBX_ERR_CUDA, cudaGetErrorString(e));
  if (st == 0) return LBX_OK;
  cudaMemset(d->tiled_flags, 0, (size_t)(ntiles + 1) * sizeof(int));
  d->tiled_base = 0;
  return lbx_internal_fail(LBX_ERR_CUDA, "tiled run: a block's wait for its neighbours ran out");
}
