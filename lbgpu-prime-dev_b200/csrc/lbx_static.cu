// lbx_static.cu -- FP64 macro-variable reductions that allocate nothing.
//
// lbx_reduce computes per-block partial sums in scratch memory that the
// domain allocates with cudaMalloc.  Some callers cannot allocate device
// memory at all: a host program whose device memory is handed in full to its
// own pool allocator, or one that must not add an allocation (which can
// synchronize the whole device, or fail) to a time-critical loop.  For them
// lbx_reduce_mv_static takes the macro variables and the mask as device
// pointers the caller owns and keeps its scratch in the fixed array below.
//
// The scratch is a file-scope __device__ array of 4097 partial sums (96 B
// each, 384 KiB): every GPU that loads this library holds it until the
// process exits.  Host code
// must not pass the array's name to a kernel -- on the host that name is
// only a stand-in, not a device address -- so the first call in each CUDA
// context looks the address up with cudaGetSymbolAddress and keeps it,
// keyed on that context (a driver-API context on a device has its own copy
// of the array, at its own address).
#include "lbx.h"
#include "lbx_kernels.cuh"

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace {

constexpr int kThreads = 256;
constexpr int kNodesPerBlock = kThreads * 64;          // 16384 nodes per partial
constexpr int kMaxPartials = 4096;                     // => at most 67,108,864 nodes
constexpr long long kMaxNodes = (long long)kNodesPerBlock * kMaxPartials;
constexpr int kMaxContexts = 64;

using lbx::RedPartial;

// Partials of one call, then the final sum in slot kMaxPartials.
static __device__ __align__(256) RedPartial g_red_scratch[kMaxPartials + 1];

// The array's device address per CUDA context, filled on first use in that
// context; guarded by g_addr_mu (two host threads may make their first calls
// at once).
struct ScratchAddr {
  void* ctx;
  RedPartial* addr;
};
ScratchAddr g_addr[kMaxContexts];
int g_naddr = 0;
std::mutex g_addr_mu;

// cuCtxGetCurrent, fetched through the runtime so that the library does not
// link the driver library itself.
typedef int (*CtxGetCurrentFn)(void**);

}  // namespace

// Defined in lbx_abi.cu, not exported: records the message lbx_last_error()
// returns on this thread.
lbx_status lbx_internal_fail(lbx_status code, const char* msg);

namespace {

lbx_status sfail(lbx_status code, const char* fmt, ...)
{
  char buf[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return lbx_internal_fail(code, buf);
}

__device__ __forceinline__ void zero(RedPartial& r)
{
  r.mass = r.solute = 0;
  for (int c = 0; c < 3; ++c) { r.mom[c] = 0; r.usum[c] = 0; }
  r.rmin = 1e300; r.rmax = -1e300; r.fluid = 0; r.nonfinite = 0;
}

__device__ __forceinline__ void combine(RedPartial& a, const RedPartial& b)
{
  a.mass += b.mass; a.solute += b.solute;
  for (int c = 0; c < 3; ++c) { a.mom[c] += b.mom[c]; a.usum[c] += b.usum[c]; }
  a.rmin = fmin(a.rmin, b.rmin); a.rmax = fmax(a.rmax, b.rmax);
  a.fluid += b.fluid; a.nonfinite += b.nonfinite;
}

__device__ void block_reduce(RedPartial& r, RedPartial* out)
{
  for (int off = 16; off > 0; off >>= 1) {
    RedPartial o;
    o.mass = __shfl_down_sync(0xffffffffu, r.mass, off);
    o.solute = __shfl_down_sync(0xffffffffu, r.solute, off);
    for (int c = 0; c < 3; ++c) {
      o.mom[c] = __shfl_down_sync(0xffffffffu, r.mom[c], off);
      o.usum[c] = __shfl_down_sync(0xffffffffu, r.usum[c], off);
    }
    o.rmin = __shfl_down_sync(0xffffffffu, r.rmin, off);
    o.rmax = __shfl_down_sync(0xffffffffu, r.rmax, off);
    o.fluid = __shfl_down_sync(0xffffffffu, r.fluid, off);
    o.nonfinite = __shfl_down_sync(0xffffffffu, r.nonfinite, off);
    combine(r, o);
  }
  __shared__ RedPartial sh[kThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    RedPartial t = sh[0];
    for (int w = 1; w < kThreads / 32; ++w) combine(t, sh[w]);
    *out = t;
  }
}

// Block b reduces nodes [b*kNodesPerBlock, (b+1)*kNodesPerBlock) into
// scratch[b]; every slot the final pass reads is written here first.
template <typename T, int D>
__global__ void __launch_bounds__(kThreads)
reduce_chunks(const T* mv, const uint8_t* solids, long long N, int nsubs, RedPartial* scratch)
{
  RedPartial r;
  zero(r);
  const long long n0 = (long long)blockIdx.x * kNodesPerBlock;
  const long long n1 = n0 + kNodesPerBlock < N ? n0 + kNodesPerBlock : N;
  for (long long n = n0 + threadIdx.x; n < n1; n += kThreads) {
    if (solids[n] == 1) continue;
    const double rho = (double)mv[n];
    const double u[3] = {(double)mv[N + n], (double)mv[2 * N + n],
                         D == 3 ? (double)mv[3 * N + n] : 0.0};
    if (!isfinite(rho) || !isfinite(u[0]) || !isfinite(u[1]) || !isfinite(u[2])) {
      r.nonfinite++;
      continue;
    }
    r.fluid++;
    r.mass += rho;
    r.rmin = fmin(r.rmin, rho);
    r.rmax = fmax(r.rmax, rho);
    for (int c = 0; c < 3; ++c) { r.mom[c] += rho * u[c]; r.usum[c] += u[c]; }
    if (nsubs == 2) r.solute += (double)mv[(long long)(1 + D) * N + n];
  }
  block_reduce(r, scratch + blockIdx.x);
}

// One block folds the partials [0, nparts) into scratch[kMaxPartials].
__global__ void __launch_bounds__(kThreads)
reduce_partials(RedPartial* scratch, int nparts)
{
  RedPartial r;
  zero(r);
  for (int b = threadIdx.x; b < nparts; b += kThreads) combine(r, scratch[b]);
  block_reduce(r, scratch + kMaxPartials);
}

}  // namespace

extern "C" lbx_status lbx_reduce_mv_static(const void* mv, const uint8_t* solids,
                                           long long N, int dims, int nsubs, int precision,
                                           void* stream, lbx_reductions* out)
{
  if (!mv || !solids || !out) return sfail(LBX_ERR_INVALID, "NULL argument");
  if (dims != 2 && dims != 3) return sfail(LBX_ERR_INVALID, "dims must be 2 or 3");
  if (nsubs != 1 && nsubs != 2) return sfail(LBX_ERR_INVALID, "nsubs must be 1 or 2");
  if (precision != 4 && precision != 8) return sfail(LBX_ERR_INVALID, "precision must be 4 or 8");
  if (N <= 0) return sfail(LBX_ERR_INVALID, "N must be positive");
  if (N > kMaxNodes)
    return sfail(LBX_ERR_INVALID,
                 "N = %lld exceeds the %lld nodes the static scratch (%d partials of %d "
                 "nodes) covers", N, kMaxNodes, kMaxPartials, kNodesPerBlock);
  // set-up, once per context, with the caller's device current
  cudaError_t e;
  static CtxGetCurrentFn ctx_current = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      fn = nullptr;
    return (CtxGetCurrentFn)fn;
  }();
  if (!ctx_current) return sfail(LBX_ERR_CUDA, "cuCtxGetCurrent is not available");
  void* ctx = nullptr;
  if (ctx_current(&ctx) != 0) return sfail(LBX_ERR_CUDA, "cuCtxGetCurrent failed");
  if (!ctx) {
    // no context bound to this thread yet: the runtime binds the current
    // device's primary context on its first call that needs one
    RedPartial* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_red_scratch);
    if (e != cudaSuccess)
      return sfail(LBX_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    if (ctx_current(&ctx) != 0 || !ctx) return sfail(LBX_ERR_CUDA, "no current CUDA context");
  }
  RedPartial* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    for (int i = 0; i < g_naddr; ++i)
      if (g_addr[i].ctx == ctx) scratch = g_addr[i].addr;
    if (!scratch) {
      e = cudaGetSymbolAddress((void**)&scratch, g_red_scratch);
      if (e != cudaSuccess || !scratch)
        return sfail(LBX_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      if (g_naddr < kMaxContexts) g_addr[g_naddr++] = ScratchAddr{ctx, scratch};
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nparts = (int)((N + kNodesPerBlock - 1) / kNodesPerBlock);
  if (precision == 8) {
    if (dims == 2) reduce_chunks<double, 2><<<nparts, kThreads, 0, st>>>((const double*)mv, solids, N, nsubs, scratch);
    else reduce_chunks<double, 3><<<nparts, kThreads, 0, st>>>((const double*)mv, solids, N, nsubs, scratch);
  } else {
    if (dims == 2) reduce_chunks<float, 2><<<nparts, kThreads, 0, st>>>((const float*)mv, solids, N, nsubs, scratch);
    else reduce_chunks<float, 3><<<nparts, kThreads, 0, st>>>((const float*)mv, solids, N, nsubs, scratch);
  }
  reduce_partials<<<1, kThreads, 0, st>>>(scratch, nparts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return sfail(LBX_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  RedPartial h;
  e = cudaMemcpyAsync(&h, scratch + kMaxPartials, sizeof h, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sfail(LBX_ERR_CUDA, "%s", cudaGetErrorString(e));
  std::memset(out, 0, sizeof *out);
  out->mass = h.mass; out->solute_mass = h.solute;
  for (int c = 0; c < 3; ++c) { out->momentum[c] = h.mom[c]; out->u_sum[c] = h.usum[c]; }
  out->rho_min = h.rmin; out->rho_max = h.rmax;
  out->fluid_nodes = (long long)h.fluid;
  out->nonfinite = (int)h.nonfinite;
  if (h.nonfinite)
    return sfail(LBX_ERR_NUMERIC, "%llu fluid nodes hold non-finite macro variables",
                 (unsigned long long)h.nonfinite);
  return LBX_OK;
}
