// lbx_batch.cu -- many independent lattices stepped together.
//
// A batch holds samples of uneven size (same velocity set, precision and
// collision model; own extents, mask, tau, rho_A and body force) in one
// compact population array [a][Ftot].  Each sample's fluid nodes occupy a
// range starting at a multiple of kAlign, so no thread block straddles two
// samples.  The samples' order in the array is a layout (lbx_batch_set_layout):
// largest first by default, so the tail of every step is made of small
// blocks; interleaved or as given on request.
//
// Sample descriptors (extents, constants, table addresses) live in a pool in
// constant memory, written once when the batch is created: a block reads its
// sample's position from a per-block table (one 4-byte load) and the
// descriptor from the constant bank where the update uses it, so the
// per-sample values cost the thread no registers, as the single-lattice
// kernels' arguments do.  A batch whose descriptors do not fit the pool's
// free space reads them from a per-block table in global memory instead.
//
// Modes (lbx_batch_run):
//   FUSED       one launch per lattice step covering every sample; runs of
//               steps are replayed from a captured CUDA graph;
//   PERSISTENT  one cooperative launch per run of steps: a grid of resident
//               blocks walks all sample blocks, with a grid-wide barrier
//               between steps (the AA pattern needs the odd step complete
//               before the even one);
//   SEQUENTIAL  one launch per sample per step (the per-sample baseline).
// lbx_batch_autotune times FUSED at each block size and PERSISTENT with the
// full and half resident grid, in each sample order, on a few steps and
// keeps the fastest.
#include "lbx.h"
#include "lbx_internal.h"
#include "lbx_kernels.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <type_traits>
#include <vector>

namespace cg = cooperative_groups;
using namespace lbx;


namespace {

constexpr int kAlign = 512;   // sample ranges start at multiples of this

lbx_status bfail(lbx_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return lbx_internal_fail(code, buf);
}

template <typename T>
struct alignas(16) SampleDesc {
  const uint2* frm;     // the sample's rank table, word 0 (device)
  T* mv;                // the sample's macro variables [1+D][N] (device)
  long long N;          // dense nodes
  int LX, LY, LZ;
  int cbase;            // first compact index (a multiple of kAlign)
  int F;                // fluid nodes
  FastDiv div_plane, div_lx;
  SubsConst<T> sc;
};

// The descriptor pool (one per device, as constant memory is).  A batch's
// range holds its descriptors in layout order.
constexpr int kPoolBytes = 63 * 1024;
__constant__ __align__(16) unsigned char g_pool[kPoolBytes];

struct PoolRef {
  int desc;             // byte offset of the descriptors in g_pool
  int block0;           // the launch's first block in the batch
};

template <typename T>
struct BatchArgs {
  T* f;                         // [Q][Ftot]
  T* mv;                        // per sample [1+D][N]
  const uint2* frm;             // per sample, ceil(N/32) words: (global compact index
                                // of the word's first fluid node, fluid bits)
  const int* fnode;             // [Ftot]: dense index inside the sample, -1 padding
  const SampleDesc<T>* blkdesc; // [nblocks]: the descriptor of each block's sample
                                // (global-memory path)
  const int* blkpos;            // [nblocks]: the layout position of each block's
                                // sample (pool path)
  long long Ftot;
  int nblocks;                  // blocks of the current block size
  int block0;                   // first block (SEQUENTIAL mode, global-memory path)
  int write_mv;
  int kahan;                    // compensated density sums
};

// One block of the batch: the single-lattice compact update (compact_node,
// with its rank-table neighbour lookups and pull-slot table) on the block's
// sample: its extents, constants and rank table, whose word ranks are
// global compact indices, so the neighbours it finds are slots of the
// shared population array.
// An even step also updates the
// padding slots after a sample, in place like any node's own slots: no real
// node ever reads them, so whatever values they take never reach a sample,
// and the step's population loads need not wait for the descriptor.  An odd
// step (whose neighbour lookups need a real node) and a step writing the
// macro variables skip the padding.
template <typename T, int Q, int MODEL, bool ODD, bool IDX32>
__device__ __forceinline__ void batch_node(const SampleDesc<T>& S, const BatchArgs<T>& A,
                                           const int m)
{
  if ((ODD || A.write_mv) && m - S.cbase >= S.F) return;   // padding after the sample
  CompactArgs<T> C;
  StepArgs<T>& L = C.s;
  L.f = A.f;
  L.mv = S.mv;
  L.LX = S.LX; L.LY = S.LY; L.LZ = S.LZ;
  L.N = S.N;
  L.sc[0] = S.sc;
  L.write_mv = A.write_mv;
  L.kahan = A.kahan;
  L.solute_on = 0;
  L.btc = nullptr;
  L.ubuf = nullptr;
  L.fout = nullptr;
  L.ns = nullptr;
  C.fnode = A.fnode;
  C.frm = S.frm;
  C.F = S.cbase + S.F;
  C.P = (int)A.Ftot;
  C.div_plane = S.div_plane;
  C.div_lx = S.div_lx;
  C.faces = 0;
  compact_node<T, Q, 1, MODEL, ODD, PART_ALL, IDX32, false>(C, m);
}

// Global-memory path: the block's descriptor from the per-block table, one
// load that depends only on the block index.
template <typename T, int Q, int MODEL, bool ODD, bool IDX32>
__device__ __forceinline__ void batch_block(const BatchArgs<T>& A, int b)
{
  batch_node<T, Q, MODEL, ODD, IDX32>(A.blkdesc[b], A, b * blockDim.x + threadIdx.x);
}

// Up to 256 threads per block, resident blocks as for the single-lattice
// compact kernels.
template <typename T, int Q, int MODEL, bool ODD, bool IDX32>
__global__ void __launch_bounds__(256, (compact_min_blocks<T, PART_ALL>()))
aa_step_batch(BatchArgs<T> A)
{
  batch_block<T, Q, MODEL, ODD, IDX32>(A, A.block0 + blockIdx.x);
}

// Pool path: the block's sample position from the per-block table, its
// descriptor from the pool.  (A binary search of the samples' first blocks
// in the pool instead cost the odd step 3-6 %: nine dependent constant-cache
// reads that miss when 512 samples' tables share an SM's constant cache.)
template <typename T, int Q, int MODEL, bool ODD, bool IDX32>
__global__ void __launch_bounds__(256, (compact_min_blocks<T, PART_ALL>()))
aa_step_batch_pool(BatchArgs<T> A, PoolRef R)
{
  const int bl = R.block0 + blockIdx.x;
  const int pos = __ldg(A.blkpos + bl);
  const SampleDesc<T>* desc = reinterpret_cast<const SampleDesc<T>*>(g_pool + R.desc);
  batch_node<T, Q, MODEL, ODD, IDX32>(desc[pos], A, bl * blockDim.x + threadIdx.x);
}

// Persistent: a resident grid walks all blocks of the batch for `steps`
// lattice steps starting at parity `odd0`, with a grid barrier between steps.
template <typename T, int Q, int MODEL, bool IDX32>
__global__ void __launch_bounds__(256)
aa_run_batch_persistent(BatchArgs<T> A, int steps, int odd0)
{
  cg::grid_group g = cg::this_grid();
  for (int st = 0; st < steps; ++st) {
    const bool odd = ((odd0 + st) & 1) != 0;
    for (int b = blockIdx.x; b < A.nblocks; b += gridDim.x) {
      if (odd) batch_block<T, Q, MODEL, true, IDX32>(A, b);
      else batch_block<T, Q, MODEL, false, IDX32>(A, b);
    }
    g.sync();
  }
}

template <typename T>
__global__ void batch_gather(T* fc, const T* fdense, const int* fnode, long long Ftot, int Q,
                             int cbase, int F, long long N)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)F * Q) return;
  const int a = (int)(t / F), ml = (int)(t - (long long)a * F);
  fc[a * Ftot + cbase + ml] = fdense[a * N + fnode[cbase + ml]];
}

template <typename T>
__global__ void batch_scatter(T* fdense, const T* fc, const int* fnode, long long Ftot, int Q,
                              int cbase, int F, long long N)
{
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)F * Q) return;
  const int a = (int)(t / F), ml = (int)(t - (long long)a * F);
  fdense[a * N + fnode[cbase + ml]] = fc[a * Ftot + cbase + ml];
}

}  // namespace

struct lbx_batch {
  int nsamples = 0, dims = 0, Q = 0, precision = 0, model = 0, kahan = 0;
  std::vector<lbx_params> params;         // per sample (as given)
  std::vector<long long> N, dbase, fbase_dense, mvbase, frm_base;
  std::vector<int> cbase, F, order;
  long long Ntot = 0, Ftot = 0;
  void* fc = nullptr;         // [Q][Ftot]
  void* fdense = nullptr;     // per sample [Q][N]: the exchange format
  void* mv = nullptr;
  uint2* frm = nullptr;       // per-sample rank tables (BatchArgs::frm)
  int* fnode = nullptr;
  uint8_t* solids = nullptr;
  void* blkdesc[2] = {nullptr, nullptr};   // SampleDesc<real> per block, block sizes 128, 256
  int* blkpos[2] = {nullptr, nullptr};     // sample position per block, block sizes 128, 256
  int device = 0;
  int layout = LBX_BATCH_LAYOUT_LARGEST_FIRST;   // sample order of the compact array
  long long frm_words = 0;    // rank-table words, guards included
  int pool_off = -1;          // the batch's range in g_pool (bytes), -1: none
  int pool_len = 0;
  int pool_desc = 0;          // offset of the descriptors in g_pool
  int nblocks[2] = {0, 0};
  void* red = nullptr;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  int parity = 0;
  int mode = LBX_BATCH_FUSED;
  int bs_index = 1;           // block size 256
  bool dense_stale = false;
  long long launches = 0;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t graph_stream = nullptr;
  int graph_bs = -1;
  int coop_grid = 0;           // resident blocks of the persistent kernel
  int coop_div = 1;            // persistent grid = coop_grid / coop_div (autotuned)
};

namespace {

const int kBlockSizes[2] = {128, 256};
constexpr int kNumBlockSizes = 2;

template <typename T, int Q, int MODEL>
BatchArgs<T> batch_args(lbx_batch* b, int write_mv)
{
  BatchArgs<T> A;
  std::memset(&A, 0, sizeof A);
  A.f = (T*)b->fc; A.mv = (T*)b->mv; A.frm = b->frm; A.fnode = b->fnode;
  A.blkdesc = (const SampleDesc<T>*)b->blkdesc[b->bs_index];
  A.blkpos = b->blkpos[b->bs_index];
  A.Ftot = b->Ftot; A.nblocks = b->nblocks[b->bs_index];
  A.write_mv = write_mv;
  A.kahan = b->kahan;
  return A;
}

template <typename T, int Q, int MODEL>
lbx_status launch_step(lbx_batch* b, bool odd, int write_mv, int mode)
{
  BatchArgs<T> A = batch_args<T, Q, MODEL>(b, write_mv);
  const int bs = kBlockSizes[b->bs_index];
  const bool idx32 = (unsigned long long)Q * (unsigned long long)b->Ftot < (1ull << 32);
  auto go_pool = [&](unsigned nb, const PoolRef& R) {
    if (idx32) {
      if (odd) aa_step_batch_pool<T, Q, MODEL, true, true><<<nb, bs, 0, b->stream>>>(A, R);
      else aa_step_batch_pool<T, Q, MODEL, false, true><<<nb, bs, 0, b->stream>>>(A, R);
    } else {
      if (odd) aa_step_batch_pool<T, Q, MODEL, true, false><<<nb, bs, 0, b->stream>>>(A, R);
      else aa_step_batch_pool<T, Q, MODEL, false, false><<<nb, bs, 0, b->stream>>>(A, R);
    }
    b->launches++;
  };
  auto go_global = [&](unsigned nb) {
    if (idx32) {
      if (odd) aa_step_batch<T, Q, MODEL, true, true><<<nb, bs, 0, b->stream>>>(A);
      else aa_step_batch<T, Q, MODEL, false, true><<<nb, bs, 0, b->stream>>>(A);
    } else {
      if (odd) aa_step_batch<T, Q, MODEL, true, false><<<nb, bs, 0, b->stream>>>(A);
      else aa_step_batch<T, Q, MODEL, false, false><<<nb, bs, 0, b->stream>>>(A);
    }
    b->launches++;
  };
  const bool pool = b->pool_off >= 0;
  PoolRef R;
  R.desc = b->pool_desc;
  if (mode == LBX_BATCH_SEQUENTIAL) {
    for (int i = 0; i < b->nsamples; ++i) {
      const int s = b->order[i];
      if (b->F[s] == 0) continue;
      const unsigned nb = (unsigned)((b->F[s] + bs - 1) / bs);
      if (pool) {
        R.block0 = b->cbase[s] / bs;
        go_pool(nb, R);
      } else {
        A.block0 = b->cbase[s] / bs;
        go_global(nb);
      }
    }
  } else if (A.nblocks > 0) {
    if (pool) {
      R.block0 = 0;
      go_pool((unsigned)A.nblocks, R);
    } else {
      go_global((unsigned)A.nblocks);
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(LBX_ERR_CUDA, "batch step: %s", cudaGetErrorString(e));
  return LBX_OK;
}

template <typename T, int Q, int MODEL>
lbx_status launch_persistent(lbx_batch* b, int steps, bool odd_first)
{
  BatchArgs<T> A = batch_args<T, Q, MODEL>(b, 0);
  // the persistent kernel is compiled for 256-thread blocks
  A.blkdesc = (const SampleDesc<T>*)b->blkdesc[1];
  A.nblocks = b->nblocks[1];
  const bool idx32 = (unsigned long long)Q * (unsigned long long)b->Ftot < (1ull << 32);
  if (b->coop_grid == 0) {
    int dev = 0, sms = 0, per_sm = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, idx32 ? (const void*)aa_run_batch_persistent<T, Q, MODEL, true>
                       : (const void*)aa_run_batch_persistent<T, Q, MODEL, false>, 256, 0);
    if (e != cudaSuccess || !coop || per_sm < 1)
      return bfail(LBX_ERR_CUDA, "persistent mode unavailable (%s)", cudaGetErrorString(e));
    b->coop_grid = sms * per_sm;
  }
  const int grid = std::min(std::max(1, b->coop_grid / b->coop_div), std::max(1, A.nblocks));
  int odd0 = odd_first ? 1 : 0;
  void* args[] = {&A, &steps, &odd0};
  cudaError_t e = cudaLaunchCooperativeKernel(
      idx32 ? (const void*)aa_run_batch_persistent<T, Q, MODEL, true>
            : (const void*)aa_run_batch_persistent<T, Q, MODEL, false>,
      grid, 256, args, 0, b->stream);
  if (e != cudaSuccess) return bfail(LBX_ERR_CUDA, "persistent launch: %s", cudaGetErrorString(e));
  b->launches++;
  return LBX_OK;
}

template <typename T, int Q>
lbx_status dispatch_step(lbx_batch* b, bool odd, int write_mv, int mode)
{
  if (b->model == SHIFTED_INC) return launch_step<T, Q, SHIFTED_INC>(b, odd, write_mv, mode);
  if (b->model == PLAIN_COMP) return launch_step<T, Q, PLAIN_COMP>(b, odd, write_mv, mode);
  return launch_step<T, Q, SHIFTED_COMP>(b, odd, write_mv, mode);
}

template <typename T, int Q>
lbx_status dispatch_persistent(lbx_batch* b, int steps, bool odd_first)
{
  if (b->model == SHIFTED_INC) return launch_persistent<T, Q, SHIFTED_INC>(b, steps, odd_first);
  if (b->model == PLAIN_COMP) return launch_persistent<T, Q, PLAIN_COMP>(b, steps, odd_first);
  return launch_persistent<T, Q, SHIFTED_COMP>(b, steps, odd_first);
}

lbx_status step_one(lbx_batch* b, bool odd, int write_mv, int mode)
{
  if (b->precision == 8)
    return b->Q == 9 ? dispatch_step<double, 9>(b, odd, write_mv, mode)
                     : dispatch_step<double, 19>(b, odd, write_mv, mode);
  return b->Q == 9 ? dispatch_step<float, 9>(b, odd, write_mv, mode)
                   : dispatch_step<float, 19>(b, odd, write_mv, mode);
}

lbx_status persistent_run(lbx_batch* b, int steps, bool odd_first)
{
  if (b->precision == 8)
    return b->Q == 9 ? dispatch_persistent<double, 9>(b, steps, odd_first)
                     : dispatch_persistent<double, 19>(b, steps, odd_first);
  return b->Q == 9 ? dispatch_persistent<float, 9>(b, steps, odd_first)
                   : dispatch_persistent<float, 19>(b, steps, odd_first);
}

template <typename T>
void fill_desc(lbx_batch* b, std::vector<unsigned char>& out)
{
  std::vector<SampleDesc<T>> d(b->nsamples);
  for (int s = 0; s < b->nsamples; ++s) {
    const lbx_params& p = b->params[s];
    SampleDesc<T>& x = d[s];
    std::memset(&x, 0, sizeof x);
    x.LX = p.LX; x.LY = p.LY; x.LZ = p.LZ;
    x.N = b->N[s];
    x.cbase = b->cbase[s]; x.F = b->F[s];
    x.frm = b->frm + b->frm_base[s];
    x.mv = (T*)b->mv + b->mvbase[s];
    x.div_plane = make_fastdiv((unsigned)(p.LX * p.LY));
    x.div_lx = make_fastdiv((unsigned)p.LX);
    const T tau = (T)p.tau[0];
    const T itau = (T)(1. / tau);
    x.sc.itau = itau; x.sc.omc = (T)(1. - itau); x.sc.rhoA = (T)p.rho_A[0];
    for (int c = 0; c < 3; ++c) x.sc.tg[c] = tau * (T)p.gaccel[c];
  }
  out.resize(d.size() * sizeof(SampleDesc<T>));
  std::memcpy(out.data(), d.data(), out.size());
}

// g_pool's ranges in use on each device: (offset, length), sorted.
constexpr int kPoolDevices = 64;
std::mutex g_pool_mu;
std::vector<std::pair<int, int>> g_pool_used[kPoolDevices];

// First fit of `len` bytes (a multiple of 16) on `dev`; -1 when none is free.
int pool_claim(int dev, int len)
{
  if (dev < 0 || dev >= kPoolDevices || len <= 0 || len > kPoolBytes) return -1;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  std::vector<std::pair<int, int>>& used = g_pool_used[dev];
  int at = 0;
  size_t i = 0;
  for (; i < used.size(); ++i) {
    if (used[i].first - at >= len) break;
    at = used[i].first + used[i].second;
  }
  if (i == used.size() && kPoolBytes - at < len) return -1;
  used.insert(used.begin() + (long)i, std::make_pair(at, len));
  return at;
}

void pool_release(int dev, int off)
{
  if (off < 0 || dev < 0 || dev >= kPoolDevices) return;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  std::vector<std::pair<int, int>>& used = g_pool_used[dev];
  for (size_t i = 0; i < used.size(); ++i)
    if (used[i].first == off) { used.erase(used.begin() + (long)i); return; }
}

// The batch's pool range: its descriptors in layout order.  Leaves pool_off
// at -1 (the global-memory path) when the pool has no room.
template <typename T>
cudaError_t pool_fill(lbx_batch* b, const std::vector<unsigned char>& desc)
{
  const int n = b->nsamples;
  const long long len = ((long long)n * (long long)sizeof(SampleDesc<T>) + 15) / 16 * 16;
  if (len > kPoolBytes) return cudaSuccess;
  const int off = pool_claim(b->device, (int)len);
  if (off < 0) return cudaSuccess;
  std::vector<unsigned char> img((size_t)len, 0);
  for (int i = 0; i < n; ++i)
    std::memcpy(img.data() + (size_t)i * sizeof(SampleDesc<T>),
                desc.data() + (size_t)b->order[i] * sizeof(SampleDesc<T>), sizeof(SampleDesc<T>));
  cudaError_t e = cudaMemcpyToSymbol(g_pool, img.data(), (size_t)len, (size_t)off,
                                     cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { pool_release(b->device, off); return e; }
  b->pool_off = off;
  b->pool_len = (int)len;
  b->pool_desc = off;
  return cudaSuccess;
}

void release(lbx_batch* b)
{
  if (b->graph) cudaGraphExecDestroy(b->graph);
  cudaFree(b->fc); cudaFree(b->fdense); cudaFree(b->mv); cudaFree(b->frm);
  cudaFree(b->fnode); cudaFree(b->solids); cudaFree(b->red);
  for (int i = 0; i < kNumBlockSizes; ++i) { cudaFree(b->blkdesc[i]); cudaFree(b->blkpos[i]); }
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  pool_release(b->device, b->pool_off);
  b->pool_off = -1;
}

lbx_status exchange(lbx_batch* b, int s, bool to_compact)
{
  if (b->F[s] == 0) return LBX_OK;
  const long long total = (long long)b->F[s] * b->Q;
  const unsigned nb = (unsigned)((total + 255) / 256);
  const size_t rs = (size_t)b->precision;
  char* fd = (char*)b->fdense + (size_t)b->fbase_dense[s] * rs;
  if (b->precision == 8) {
    if (to_compact) batch_gather<double><<<nb, 256, 0, b->stream>>>((double*)b->fc, (const double*)fd, b->fnode, b->Ftot, b->Q, b->cbase[s], b->F[s], b->N[s]);
    else batch_scatter<double><<<nb, 256, 0, b->stream>>>((double*)fd, (const double*)b->fc, b->fnode, b->Ftot, b->Q, b->cbase[s], b->F[s], b->N[s]);
  } else {
    if (to_compact) batch_gather<float><<<nb, 256, 0, b->stream>>>((float*)b->fc, (const float*)fd, b->fnode, b->Ftot, b->Q, b->cbase[s], b->F[s], b->N[s]);
    else batch_scatter<float><<<nb, 256, 0, b->stream>>>((float*)fd, (const float*)b->fc, b->fnode, b->Ftot, b->Q, b->cbase[s], b->F[s], b->N[s]);
  }
  b->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(LBX_ERR_CUDA, "batch exchange: %s", cudaGetErrorString(e));
  return LBX_OK;
}

lbx_status sync_dense(lbx_batch* b)
{
  if (!b->dense_stale) return LBX_OK;
  for (int s = 0; s < b->nsamples; ++s)
    if (lbx_status st = exchange(b, s, false)) return st;
  b->dense_stale = false;
  return LBX_OK;
}

lbx_status check_sample(lbx_batch* b, int s)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  if (s < 0 || s >= b->nsamples) return bfail(LBX_ERR_INVALID, "sample %d out of range", s);
  return LBX_OK;
}

#define BCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return bfail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,       \
                   "%s: %s", #call, cudaGetErrorString(e_));                             \
  } while (0)

// Replay `pairs` AA pairs (FUSED mode) from one captured pair.
lbx_status fused_pairs(lbx_batch* b, int pairs)
{
  if (!b->graph || b->graph_stream != b->stream || b->graph_bs != b->bs_index) {
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const long long before = b->launches;
    lbx_status st = step_one(b, true, 0, LBX_BATCH_FUSED);
    if (st == LBX_OK) st = step_one(b, false, 0, LBX_BATCH_FUSED);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->launches = before;
    if (st != LBX_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return bfail(LBX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->graph = nullptr; return bfail(LBX_ERR_CUDA, "graph: %s", cudaGetErrorString(e)); }
    b->graph_stream = b->stream;
    b->graph_bs = b->bs_index;
  }
  for (int r = 0; r < pairs; ++r) {
    BCK(cudaGraphLaunch(b->graph, b->stream));
    b->launches += 2;
  }
  return LBX_OK;
}

lbx_status run_steps(lbx_batch* b, int t0, int nsteps, int frame_rate, int mode)
{
  int t = t0 + 1;
  const int tend = t0 + nsteps;
  while (t <= tend) {
    const bool odd = (t % 2) != 0;
    if (odd != (b->parity == 0))
      return bfail(LBX_ERR_STATE, "batch step at time %d out of AA order", t);
    // frame-free stretch
    int stretch = 0;
    while (t + stretch <= tend && !(frame_rate > 0 && (t + stretch) % frame_rate == 0)) ++stretch;
    if (mode == LBX_BATCH_PERSISTENT && stretch >= 2) {
      if (lbx_status st = persistent_run(b, stretch, odd)) return st;
      b->parity ^= (stretch & 1);
      t += stretch;
      continue;
    }
    if (mode == LBX_BATCH_FUSED && odd && stretch >= 4 && b->stream != nullptr) {
      const int pairs = stretch / 2;
      if (lbx_status st = fused_pairs(b, pairs)) return st;
      t += 2 * pairs;
      continue;
    }
    const bool frame = frame_rate > 0 && t % frame_rate == 0;
    const int m = (mode == LBX_BATCH_SEQUENTIAL) ? LBX_BATCH_SEQUENTIAL : LBX_BATCH_FUSED;
    if (lbx_status st = step_one(b, odd, frame ? 1 : 0, m)) return st;
    b->parity ^= 1;
    ++t;
  }
  b->dense_stale = true;
  return LBX_OK;
}

}  // namespace

extern "C" {

namespace {

// The compact layout for the sample order `layout`: each sample's range in
// the population array, the dense index of every compact slot, the rank
// tables (whose ranks are global compact indices), the sample descriptors
// (pool and per-block tables).  `sol`: every sample's solids in sample order.
// The populations are not moved (lbx_batch_set_layout moves them).
lbx_status lay_out(lbx_batch* b, int layout, const std::vector<uint8_t>& sol)
{
  const int ns = b->nsamples;
  b->order.resize(ns);
  std::iota(b->order.begin(), b->order.end(), 0);
  if (layout != LBX_BATCH_LAYOUT_GIVEN) {
    // largest first: the last blocks of a step are the small ones
    std::stable_sort(b->order.begin(), b->order.end(),
                     [&](int x, int y) { return b->F[x] > b->F[y]; });
    if (layout == LBX_BATCH_LAYOUT_INTERLEAVED) {
      // largest, smallest, second largest, second smallest, ...
      std::vector<int> by_size = b->order;
      for (int i = 0, lo = 0, hi = ns - 1; i < ns; ++i)
        b->order[i] = (i & 1) ? by_size[hi--] : by_size[lo++];
    }
  }
  long long c = 0;
  for (int s : b->order) {
    b->cbase[s] = (int)c;
    c += (b->F[s] + kAlign - 1) / kAlign * kAlign;
  }
  std::vector<int> fnode(std::max<long long>(b->Ftot, 1), -1);
  std::vector<uint2> frm((size_t)b->frm_words);
  for (int s = 0; s < ns; ++s) {
    int m = b->cbase[s];
    const long long W = (b->N[s] + 31) / 32;
    uint2* tab = frm.data() + b->frm_base[s];
    tab[-1] = make_uint2((unsigned)m, 0u);
    for (long long w = 0; w < W; ++w) {
      unsigned bits = 0;
      tab[w].x = (unsigned)m;
      for (int q = 0; q < 32; ++q) {
        const long long n = w * 32 + q;
        if (n >= b->N[s]) break;
        if (sol[b->dbase[s] + n] != 1) { bits |= 1u << q; fnode[m++] = (int)n; }
      }
      tab[w].y = bits;
    }
    tab[W] = make_uint2((unsigned)m, 0u);
  }
  BCK(cudaMemcpy(b->frm, frm.data(), frm.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->fnode, fnode.data(), fnode.size() * sizeof(int), cudaMemcpyHostToDevice));
  std::vector<unsigned char> desc;   // per sample
  if (b->precision == 8) fill_desc<double>(b, desc); else fill_desc<float>(b, desc);
  const size_t dsz = desc.size() / (size_t)ns;
  pool_release(b->device, b->pool_off);
  b->pool_off = -1;
  BCK(b->precision == 8 ? pool_fill<double>(b, desc) : pool_fill<float>(b, desc));
  for (int i = 0; i < kNumBlockSizes; ++i) {
    // every block of a sample's padded range belongs to that sample and
    // holds a copy of its descriptor; a padding thread finds m - cbase >= F
    const int bs = kBlockSizes[i];
    const int nb = (int)(b->Ftot / bs);
    std::vector<unsigned char> tab((size_t)std::max(nb, 1) * dsz, 0);
    for (int s : b->order) {
      const long long len = (b->F[s] + kAlign - 1) / kAlign * kAlign;
      for (long long q = b->cbase[s] / bs; q < (b->cbase[s] + len) / bs; ++q)
        std::memcpy(tab.data() + (size_t)q * dsz, desc.data() + (size_t)s * dsz, dsz);
    }
    b->nblocks[i] = nb;
    if (!b->blkdesc[i]) BCK(cudaMalloc(&b->blkdesc[i], tab.size()));
    BCK(cudaMemcpy(b->blkdesc[i], tab.data(), tab.size(), cudaMemcpyHostToDevice));
    // the sample position of every block (the pool path's lookup)
    std::vector<int> pos((size_t)std::max(nb, 1), 0);
    for (int li = 0; li < ns; ++li) {
      const int s = b->order[li];
      const long long len = (b->F[s] + kAlign - 1) / kAlign * kAlign;
      for (long long q = b->cbase[s] / bs; q < (b->cbase[s] + len) / bs; ++q) pos[(size_t)q] = li;
    }
    if (!b->blkpos[i]) BCK(cudaMalloc(&b->blkpos[i], pos.size() * sizeof(int)));
    BCK(cudaMemcpy(b->blkpos[i], pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  // captured steps hold the old tables' launch arguments
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  b->layout = layout;
  return LBX_OK;
}

// Another sample order with the state kept: the populations go to the
// dense exchange array, the tables are rebuilt, the populations come back.
lbx_status relayout(lbx_batch* b, int layout)
{
  if (lbx_status st = sync_dense(b)) return st;
  std::vector<uint8_t> sol((size_t)b->Ntot);
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaMemcpy(sol.data(), b->solids, sol.size(), cudaMemcpyDeviceToHost));
  if (lbx_status st = lay_out(b, layout, sol)) return st;
  for (int s = 0; s < b->nsamples; ++s)
    if (lbx_status st = exchange(b, s, true)) return st;
  BCK(cudaStreamSynchronize(b->stream));
  b->dense_stale = false;
  return LBX_OK;
}

}  // namespace

lbx_status lbx_batch_create(int nsamples, const lbx_params* params, const uint8_t* const* solids,
                            lbx_batch** out)
{
  if (!out || !params || !solids || nsamples < 1)
    return bfail(LBX_ERR_INVALID, "need nsamples >= 1, params, solids and out");
  *out = nullptr;
  const lbx_params& p0 = params[0];
  for (int s = 0; s < nsamples; ++s) {
    const lbx_params& p = params[s];
    if (p.dims != p0.dims || p.precision != p0.precision || p.accurate != p0.accurate ||
        p.compressible != p0.compressible || (p.kahan != 0) != (p0.kahan != 0))
      return bfail(LBX_ERR_INVALID,
                   "sample %d: dims, precision, model and kahan must match sample 0", s);
    if ((p.dims != 2 && p.dims != 3) || p.LX < 1 || p.LY < 1 || p.LZ < 1 ||
        (p.dims == 2 && p.LZ != 1))
      return bfail(LBX_ERR_INVALID, "sample %d: bad extents", s);
    if (p.nsubs != 1) return bfail(LBX_ERR_INVALID, "sample %d: batches hold one substance", s);
    if (p.walsh) return bfail(LBX_ERR_INVALID, "sample %d: batches take no Walsh runs", s);
    if (p.precision != 4 && p.precision != 8) return bfail(LBX_ERR_INVALID, "bad precision");
    if (!p.accurate && !p.compressible) return bfail(LBX_ERR_INVALID, "accurate=0 needs compressible=1");
    if (!(p.tau[0] > 0.5)) return bfail(LBX_ERR_INVALID, "sample %d: tau must exceed 0.5", s);
    if (p.pressure_n_in[0] || p.pressure_s_in[0] || p.pressure_n_out[0] || p.pressure_s_out[0] ||
        p.pressure_t_in[0] || p.pressure_b_in[0] || p.pressure_t_out[0] || p.pressure_b_out[0] ||
        p.velocity_t_in[0] || p.velocity_b_in[0] || p.velocity_t_out[0] || p.velocity_b_out[0])
      return bfail(LBX_ERR_INVALID, "sample %d: batches have no face boundaries", s);
    if ((long long)p.LX * p.LY * p.LZ >= (1LL << 31)) return bfail(LBX_ERR_INVALID, "sample too large");
    if (!solids[s]) return bfail(LBX_ERR_INVALID, "sample %d: solids is NULL", s);
  }
  BCK(cudaSetDevice(p0.device));
  lbx_batch* b = new lbx_batch();
  b->device = p0.device;
  b->nsamples = nsamples;
  b->dims = p0.dims;
  b->Q = p0.dims == 2 ? 9 : 19;
  b->precision = p0.precision;
  b->model = p0.accurate ? (p0.compressible ? SHIFTED_COMP : SHIFTED_INC) : PLAIN_COMP;
  b->kahan = p0.kahan ? 1 : 0;
  b->params.assign(params, params + nsamples);
  b->N.resize(nsamples); b->dbase.resize(nsamples); b->fbase_dense.resize(nsamples);
  b->mvbase.resize(nsamples); b->cbase.resize(nsamples); b->F.resize(nsamples);
  for (int s = 0; s < nsamples; ++s) {
    const lbx_params& p = params[s];
    b->N[s] = (long long)p.LX * p.LY * p.LZ;
    long long f = 0;
    for (long long n = 0; n < b->N[s]; ++n) f += solids[s][n] != 1;
    b->F[s] = (int)f;
  }
  long long dn = 0, mvn = 0, c = 0;
  for (int s = 0; s < nsamples; ++s) {          // dense arrays in sample order
    b->dbase[s] = dn; b->fbase_dense[s] = dn * b->Q; b->mvbase[s] = mvn;
    dn += b->N[s]; mvn += (1 + b->dims) * b->N[s];
    c += (b->F[s] + kAlign - 1) / kAlign * kAlign;
  }
  b->Ntot = dn;
  b->Ftot = c;
  if (c >= (1LL << 31)) { delete b; return bfail(LBX_ERR_INVALID, "batch holds >= 2^31 fluid nodes"); }

  // per sample: a rank table of ceil(N/32) words (global compact index of
  // the word's first fluid node, fluid bits), with a guard word in front and
  // behind (filled by lay_out)
  std::vector<uint8_t> sol(b->Ntot);
  b->frm_base.resize(nsamples);
  long long words = 0;
  for (int s = 0; s < nsamples; ++s) {
    b->frm_base[s] = words + 1;
    words += (b->N[s] + 31) / 32 + 2;
    std::memcpy(sol.data() + b->dbase[s], solids[s], (size_t)b->N[s]);
  }
  b->frm_words = words;
  b->cbase.assign(nsamples, 0);
  auto bail = [&](lbx_status st) { release(b); delete b; return st; };
  cudaError_t e;
#define BCKD(call) if ((e = (call)) != cudaSuccess) return bail(bfail(e == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e)));
  BCKD(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
  b->stream = b->own_stream;
  const size_t rs = (size_t)b->precision;
  BCKD(cudaMalloc(&b->fc, std::max<size_t>(1, (size_t)b->Q * b->Ftot * rs)));
  BCKD(cudaMalloc(&b->fdense, (size_t)b->Q * b->Ntot * rs));
  BCKD(cudaMalloc(&b->mv, (size_t)(1 + b->dims) * b->Ntot * rs));
  BCKD(cudaMalloc(&b->frm, (size_t)b->frm_words * sizeof(uint2)));
  BCKD(cudaMalloc(&b->fnode, (size_t)std::max<long long>(b->Ftot, 1) * sizeof(int)));
  BCKD(cudaMalloc(&b->solids, (size_t)b->Ntot));
  BCKD(cudaMalloc(&b->red, 2 * 148 * sizeof(RedPartial)));
  BCKD(cudaMemcpy(b->solids, sol.data(), sol.size(), cudaMemcpyHostToDevice));
  BCKD(cudaMemset(b->fc, 0, std::max<size_t>(1, (size_t)b->Q * b->Ftot * rs)));
  BCKD(cudaMemset(b->fdense, 0, (size_t)b->Q * b->Ntot * rs));
  BCKD(cudaMemset(b->mv, 0, (size_t)(1 + b->dims) * b->Ntot * rs));
  if (lbx_status st = lay_out(b, LBX_BATCH_LAYOUT_LARGEST_FIRST, sol)) return bail(st);
#undef BCKD
  *out = b;
  return LBX_OK;
}

lbx_status lbx_batch_destroy(lbx_batch* b)
{
  if (!b) return LBX_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  release(b);
  delete b;
  return LBX_OK;
}

lbx_status lbx_batch_upload_f(lbx_batch* b, int s, const void* f_host)
{
  if (lbx_status st = check_sample(b, s)) return st;
  if (!f_host) return bfail(LBX_ERR_INVALID, "f_host is NULL");
  if (lbx_status st = sync_dense(b)) return st;
  const size_t rs = (size_t)b->precision;
  BCK(cudaMemcpyAsync((char*)b->fdense + (size_t)b->fbase_dense[s] * rs, f_host,
                      (size_t)b->Q * b->N[s] * rs, cudaMemcpyHostToDevice, b->stream));
  if (lbx_status st = exchange(b, s, true)) return st;
  BCK(cudaStreamSynchronize(b->stream));
  b->parity = 0;
  return LBX_OK;
}

lbx_status lbx_batch_download_f(lbx_batch* b, int s, void* f_host)
{
  if (lbx_status st = check_sample(b, s)) return st;
  if (!f_host) return bfail(LBX_ERR_INVALID, "f_host is NULL");
  if (lbx_status st = sync_dense(b)) return st;
  const size_t rs = (size_t)b->precision;
  BCK(cudaMemcpyAsync(f_host, (char*)b->fdense + (size_t)b->fbase_dense[s] * rs,
                      (size_t)b->Q * b->N[s] * rs, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return LBX_OK;
}

lbx_status lbx_batch_init_equilibrium(lbx_batch* b, int s, const void* rho, const void* ux,
                                      const void* uy, const void* uz)
{
  if (lbx_status st = check_sample(b, s)) return st;
  if (!rho || !ux || !uy || (b->dims == 3 && !uz))
    return bfail(LBX_ERR_INVALID, "rho/ux/uy (and uz in 3D) are required");
  if (lbx_status st = sync_dense(b)) return st;
  const size_t rs = (size_t)b->precision, plane = (size_t)b->N[s] * rs;
  void* tmp = nullptr;
  BCK(cudaMalloc(&tmp, 4 * plane));
  const void* src[4] = {rho, ux, uy, uz};
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < 4 && e == cudaSuccess; ++c)
    if (src[c]) e = cudaMemcpyAsync((char*)tmp + c * plane, src[c], plane, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) {
    const int shifted = b->model != PLAIN_COMP;
    const unsigned nb = (unsigned)((b->N[s] + 255) / 256);
    char* t = (char*)tmp;
    char* fd = (char*)b->fdense + (size_t)b->fbase_dense[s] * rs;
    if (b->precision == 8) {
      const double* uzp = uz ? (const double*)(t + 3 * plane) : nullptr;
      if (b->Q == 9) init_feq<double, 9><<<nb, 256, 0, b->stream>>>((double*)fd, (double*)t, (double*)(t + plane), (double*)(t + 2 * plane), uzp, b->N[s], shifted);
      else init_feq<double, 19><<<nb, 256, 0, b->stream>>>((double*)fd, (double*)t, (double*)(t + plane), (double*)(t + 2 * plane), uzp, b->N[s], shifted);
    } else {
      const float* uzp = uz ? (const float*)(t + 3 * plane) : nullptr;
      if (b->Q == 9) init_feq<float, 9><<<nb, 256, 0, b->stream>>>((float*)fd, (float*)t, (float*)(t + plane), (float*)(t + 2 * plane), uzp, b->N[s], shifted);
      else init_feq<float, 19><<<nb, 256, 0, b->stream>>>((float*)fd, (float*)t, (float*)(t + plane), (float*)(t + 2 * plane), uzp, b->N[s], shifted);
    }
    b->launches++;
    e = cudaGetLastError();
  }
  lbx_status st = LBX_OK;
  if (e == cudaSuccess) st = exchange(b, s, true);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return bfail(LBX_ERR_CUDA, "batch init: %s", cudaGetErrorString(e));
  b->parity = 0;
  return st;
}

lbx_status lbx_batch_download_mv(lbx_batch* b, int s, void* rho, void* ux, void* uy, void* uz)
{
  if (lbx_status st = check_sample(b, s)) return st;
  const size_t rs = (size_t)b->precision, plane = (size_t)b->N[s] * rs;
  const char* base = (const char*)b->mv + (size_t)b->mvbase[s] * rs;
  void* dst[4] = {rho, ux, uy, uz};
  for (int c = 0; c <= b->dims; ++c)
    if (dst[c]) BCK(cudaMemcpyAsync(dst[c], base + c * plane, plane, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return LBX_OK;
}

lbx_status lbx_batch_run(lbx_batch* b, int t0, int nsteps, int frame_rate, int mode)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  if (nsteps < 0) return bfail(LBX_ERR_INVALID, "nsteps must be >= 0");
  if (mode == LBX_BATCH_AUTO) mode = b->mode;
  if (mode != LBX_BATCH_FUSED && mode != LBX_BATCH_PERSISTENT && mode != LBX_BATCH_SEQUENTIAL)
    return bfail(LBX_ERR_INVALID, "unknown batch mode %d", mode);
  return run_steps(b, t0, nsteps, frame_rate, mode);
}

lbx_status lbx_batch_autotune(lbx_batch* b, int steps, int* mode_out, int* block_out)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  if (b->parity != 0) return bfail(LBX_ERR_STATE, "autotune starts from natural order");
  if (steps < 2) steps = 2;
  steps += steps & 1;
  // The trial steps advance the lattice; start from a copy and put it back.
  const size_t bytes = (size_t)b->Q * b->Ftot * (size_t)b->precision;
  const int layout0 = b->layout;
  void* save = nullptr;
  BCK(cudaMalloc(&save, std::max<size_t>(bytes, 1)));
  BCK(cudaMemcpyAsync(save, b->fc, bytes, cudaMemcpyDeviceToDevice, b->stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int best_mode = LBX_BATCH_FUSED, best_bs = 1, best_div = 1, best_layout = layout0;
  // candidates: FUSED at each block size; PERSISTENT (256-thread blocks) with
  // the resident grid, or half of it (fewer blocks contending for the grid
  // barrier, more sample blocks walked by each); each in every sample order,
  // the current one first
  struct Cand { int mode, bs, div; };
  const Cand cands[] = {{LBX_BATCH_FUSED, 0, 1}, {LBX_BATCH_FUSED, 1, 1},
                        {LBX_BATCH_PERSISTENT, 1, 1}, {LBX_BATCH_PERSISTENT, 1, 2}};
  const int layouts[3] = {layout0, (layout0 + 1) % 3, (layout0 + 2) % 3};
  lbx_status st = LBX_OK;
  for (int li = 0; li < 3 && st == LBX_OK; ++li) {
    if (layouts[li] != b->layout) st = relayout(b, layouts[li]);
    for (const Cand& c : cands) {
      if (st != LBX_OK) break;
      b->bs_index = c.bs;
      b->coop_div = c.div;
      st = run_steps(b, 0, 2, 0, c.mode);              // warm-up (and graph capture)
      if (st != LBX_OK) { st = LBX_OK; b->parity = 0; continue; }   // mode unavailable
      cudaEventRecord(e0, b->stream);
      st = run_steps(b, 2, steps, 0, c.mode);
      cudaEventRecord(e1, b->stream);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (st == LBX_OK && ms < best) {
        best = ms; best_mode = c.mode; best_bs = c.bs; best_div = c.div; best_layout = b->layout;
      }
    }
  }
  b->mode = best_mode;
  b->bs_index = best_bs;
  b->coop_div = best_div;
  b->parity = 0;
  // the saved populations are in the first order: back to it, restore, then
  // move them to the chosen order
  if (st == LBX_OK && b->layout != layout0) st = relayout(b, layout0);
  if (st == LBX_OK) {
    cudaMemcpyAsync(b->fc, save, bytes, cudaMemcpyDeviceToDevice, b->stream);
    b->dense_stale = true;
    if (best_layout != layout0) st = relayout(b, best_layout);
  }
  cudaStreamSynchronize(b->stream);
  cudaFree(save);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (mode_out) *mode_out = best_mode;
  if (block_out) *block_out = kBlockSizes[best_bs];
  return st;
}

lbx_status lbx_batch_set_layout(lbx_batch* b, int layout)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  if (layout != LBX_BATCH_LAYOUT_LARGEST_FIRST && layout != LBX_BATCH_LAYOUT_INTERLEAVED &&
      layout != LBX_BATCH_LAYOUT_GIVEN)
    return bfail(LBX_ERR_INVALID, "unknown batch layout %d", layout);
  if (layout == b->layout) return LBX_OK;
  return relayout(b, layout);
}

lbx_status lbx_batch_get_layout(lbx_batch* b, int* layout)
{
  if (!b || !layout) return bfail(LBX_ERR_INVALID, "batch and layout must not be NULL");
  *layout = b->layout;
  return LBX_OK;
}

lbx_status lbx_batch_set_stream(lbx_batch* b, void* stream)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  BCK(cudaStreamSynchronize(b->stream));
  b->stream = (cudaStream_t)stream;
  return LBX_OK;
}

lbx_status lbx_batch_sync(lbx_batch* b)
{
  if (!b) return bfail(LBX_ERR_INVALID, "batch is NULL");
  BCK(cudaStreamSynchronize(b->stream));
  BCK(cudaGetLastError());
  return LBX_OK;
}

lbx_status lbx_batch_reduce(lbx_batch* b, int s, lbx_reductions* out)
{
  if (lbx_status st = check_sample(b, s)) return st;
  if (!out) return bfail(LBX_ERR_INVALID, "out is NULL");
  const int nb = 2 * 148;
  RedPartial* red = (RedPartial*)b->red;
  const size_t rs = (size_t)b->precision;
  const void* mv = (const char*)b->mv + (size_t)b->mvbase[s] * rs;
  const uint8_t* sol = b->solids + b->dbase[s];
  if (b->precision == 8) {
    if (b->dims == 2) reduce_mv<double, 2><<<nb, 256, 0, b->stream>>>((const double*)mv, sol, b->N[s], 1, red);
    else reduce_mv<double, 3><<<nb, 256, 0, b->stream>>>((const double*)mv, sol, b->N[s], 1, red);
  } else {
    if (b->dims == 2) reduce_mv<float, 2><<<nb, 256, 0, b->stream>>>((const float*)mv, sol, b->N[s], 1, red);
    else reduce_mv<float, 3><<<nb, 256, 0, b->stream>>>((const float*)mv, sol, b->N[s], 1, red);
  }
  b->launches++;
  std::vector<RedPartial> h(nb);
  BCK(cudaMemcpyAsync(h.data(), red, nb * sizeof(RedPartial), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  std::memset(out, 0, sizeof *out);
  out->rho_min = 1e300; out->rho_max = -1e300;
  unsigned long long fl = 0, nf = 0;
  for (const RedPartial& r : h) {
    out->mass += r.mass;
    for (int c = 0; c < 3; ++c) { out->momentum[c] += r.mom[c]; out->u_sum[c] += r.usum[c]; }
    out->rho_min = std::min(out->rho_min, r.rmin); out->rho_max = std::max(out->rho_max, r.rmax);
    fl += r.fluid; nf += r.nonfinite;
  }
  out->fluid_nodes = (long long)fl;
  out->nonfinite = (int)nf;
  if (nf) return bfail(LBX_ERR_NUMERIC, "%llu non-finite macro variables", nf);
  return LBX_OK;
}

long long lbx_batch_launch_count(lbx_batch* b) { return b ? b->launches : -1; }


}  // extern "C"
