// lbx_frames.cu -- frame statistics and asynchronous frame output.
//
// The reference ends every frame with synchronous copies of the macro
// variables to the host (src/lbgpu_prime.cu:544-583, :765-804), host loops
// over every node for the frame statistics (compute_*, src/compute.c:
// 1159-1416) and the file writers.  Here the statistics are one grid-stride
// FP64 reduction on the device, and a frame is a device-side snapshot of the
// macro variables (a copy at HBM speed on the domain's stream) followed by a
// host copy on a second stream, so the steps queued after it never wait for
// the host link.
#include "lbx.h"
#include "lbx_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

namespace {

lbx_status ffail(lbx_status code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

lbx_status ffail(lbx_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return lbx_internal_fail(code, buf);
}

#define FCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return ffail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,        \
                   "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

constexpr int kThreads = 256;
constexpr int kBlocks = 2 * 148;   // two resident blocks per SM of a B200

// One block's partial statistics of one substance: channel 0 is rho,
// 1..3 are u_x, u_y, u_z.  mn starts at +inf and mx at 0.
struct FramePart {
  double sum[4];
  double mx[4];
  double mn[4];
  unsigned long long nodes;
};

// Grid-stride pass over the nodes whose mask byte is 0.  A NaN compares
// false, so it never replaces a running max or min (the reference's
// `if (u > max)` loops behave the same).  Block results are combined in a
// fixed order by frame_final, so the sums are reproducible.
template <typename T, int D>
__global__ void __launch_bounds__(kThreads)
frame_part(const T* __restrict__ mv, const uint8_t* __restrict__ mask, long long N,
           FramePart* __restrict__ part)
{
  __shared__ double s_sum[kThreads / 32][4], s_mx[kThreads / 32][4], s_mn[kThreads / 32][4];
  __shared__ unsigned long long s_cnt[kThreads / 32];
  double sum[4] = {0., 0., 0., 0.}, mx[4] = {0., 0., 0., 0.};
  double mn[4] = {HUGE_VAL, HUGE_VAL, HUGE_VAL, HUGE_VAL};
  unsigned long long cnt = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
    if (mask[n]) continue;
    ++cnt;
#pragma unroll
    for (int c = 0; c <= D; ++c) {
      const double v = (double)mv[c * N + n];
      const double a = fabs(v);
      sum[c] += v;
      if (a > mx[c]) mx[c] = a;
      if (a < mn[c]) mn[c] = a;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
#pragma unroll
    for (int c = 0; c <= D; ++c) {
      sum[c] += __shfl_down_sync(0xffffffffu, sum[c], o);
      mx[c] = fmax(mx[c], __shfl_down_sync(0xffffffffu, mx[c], o));
      mn[c] = fmin(mn[c], __shfl_down_sync(0xffffffffu, mn[c], o));
    }
  }
  if (lane == 0) {
    s_cnt[warp] = cnt;
#pragma unroll
    for (int c = 0; c < 4; ++c) { s_sum[warp][c] = sum[c]; s_mx[warp][c] = mx[c]; s_mn[warp][c] = mn[c]; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    FramePart r;
    r.nodes = 0;
    for (int c = 0; c < 4; ++c) { r.sum[c] = 0.; r.mx[c] = 0.; r.mn[c] = HUGE_VAL; }
    for (int w = 0; w < kThreads / 32; ++w) {
      r.nodes += s_cnt[w];
      for (int c = 0; c <= D; ++c) {
        r.sum[c] += s_sum[w][c];
        r.mx[c] = fmax(r.mx[c], s_mx[w][c]);
        r.mn[c] = fmin(r.mn[c], s_mn[w][c]);
      }
    }
    part[blockIdx.x] = r;
  }
}

// Combines the block partials in block order into the ABI's struct.  With
// no node counted (or only NaNs in a channel) the min equals the max, which
// is 0 -- the reference's min loops start from the max.
__global__ void frame_final(const FramePart* __restrict__ part, int nparts, int D,
                            lbx_frame_stats* __restrict__ out)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double sum[4] = {0., 0., 0., 0.}, mx[4] = {0., 0., 0., 0.};
  double mn[4] = {HUGE_VAL, HUGE_VAL, HUGE_VAL, HUGE_VAL};
  unsigned long long nodes = 0;
  for (int b = 0; b < nparts; ++b) {
    nodes += part[b].nodes;
    for (int c = 0; c < 4; ++c) {
      sum[c] += part[b].sum[c];
      mx[c] = fmax(mx[c], part[b].mx[c]);
      mn[c] = fmin(mn[c], part[b].mn[c]);
    }
  }
  for (int c = 0; c < 4; ++c) {
    if (c > D) { sum[c] = 0.; mx[c] = 0.; mn[c] = 0.; }
    if (!(mn[c] <= mx[c])) mn[c] = mx[c];
  }
  const double nn = nodes ? (double)nodes : 1.;
  out->nodes = (long long)nodes;
  out->max_rho = mx[0];
  out->min_rho = mn[0];
  out->ave_rho = nodes ? sum[0] / nn : 0.;
  for (int c = 0; c < 3; ++c) {
    out->max_u[c] = mx[1 + c];
    out->min_u[c] = mn[1 + c];
    out->ave_u[c] = nodes ? sum[1 + c] / nn : 0.;
  }
}

// Frame buffers: two slots of (device snapshot, host copy, statistics) plus
// a scratch statistics slot for lbx_frame_stats_compute.
struct Frames {
  size_t bytes = 0;                       // the macro variables of every substance
  void* snap[2] = {nullptr, nullptr};     // device snapshots, by queued % 2
  // page-locked host copies, by queued % 3: a frame's buffer is reused by the
  // third enqueue after its own, which needs its successor waited first, so
  // a returned frame's buffer outlives the first enqueue after its wait even
  // when two frames were outstanding
  void* host[3] = {nullptr, nullptr, nullptr};
  lbx_frame_stats* st_dev = nullptr;      // [3][2]: slots 0, 1 and scratch 2
  lbx_frame_stats* st_host = nullptr;     // [3][2] page-locked
  FramePart* part = nullptr;              // [kBlocks]
  cudaStream_t copy = nullptr;
  cudaEvent_t taken[2] = {nullptr, nullptr};   // snapshot and statistics queued
  cudaEvent_t landed[2] = {nullptr, nullptr};  // host copies complete
  int time[2] = {0, 0};
  int hslot[2] = {0, 0};                  // host buffer of the frame in each slot
  long long queued = 0, waited = 0;       // frames enqueued / returned
};

Frames* frames_of(lbx_domain* d)
{
  if (!d->frames) d->frames = new Frames();
  return (Frames*)d->frames;
}

// The statistics buffers, allocated on first use.
lbx_status alloc_stats(Frames* F)
{
  if (!F->part) FCK(cudaMalloc(&F->part, kBlocks * sizeof(FramePart)));
  if (!F->st_dev) FCK(cudaMalloc(&F->st_dev, 6 * sizeof(lbx_frame_stats)));
  if (!F->st_host)
    FCK(cudaHostAlloc(&F->st_host, 6 * sizeof(lbx_frame_stats), cudaHostAllocDefault));
  return LBX_OK;
}

// Statistics of substance s into st (device), queued on the domain's stream;
// the buffers of alloc_stats exist.
lbx_status queue_stats(lbx_domain* d, Frames* F, int s, lbx_frame_stats* st)
{
  const long long N = d->N;
  const size_t off = (size_t)s * (1 + d->D) * N;
  const unsigned blocks = (unsigned)std::min<long long>(kBlocks, (N + kThreads - 1) / kThreads);
  if (blocks == 0) return ffail(LBX_ERR_INVALID, "empty lattice");
  if (d->real_size == 8) {
    const double* mv = (const double*)d->mv + off;
    if (d->D == 2) frame_part<double, 2><<<blocks, kThreads, 0, d->stream>>>(mv, d->solids, N, F->part);
    else frame_part<double, 3><<<blocks, kThreads, 0, d->stream>>>(mv, d->solids, N, F->part);
  } else {
    const float* mv = (const float*)d->mv + off;
    if (d->D == 2) frame_part<float, 2><<<blocks, kThreads, 0, d->stream>>>(mv, d->solids, N, F->part);
    else frame_part<float, 3><<<blocks, kThreads, 0, d->stream>>>(mv, d->solids, N, F->part);
  }
  frame_final<<<1, 32, 0, d->stream>>>(F->part, (int)blocks, d->D, st);
  d->launches += 2;
  FCK(cudaGetLastError());
  return LBX_OK;
}

}  // namespace

void lbx_internal_frames_free(lbx_domain* d)
{
  Frames* F = (Frames*)d->frames;
  if (!F) return;
  if (F->copy) cudaStreamSynchronize(F->copy);
  for (int k = 0; k < 2; ++k) {
    cudaFree(F->snap[k]);
    if (F->taken[k]) cudaEventDestroy(F->taken[k]);
    if (F->landed[k]) cudaEventDestroy(F->landed[k]);
  }
  for (int k = 0; k < 3; ++k) cudaFreeHost(F->host[k]);
  cudaFree(F->st_dev);
  cudaFreeHost(F->st_host);
  cudaFree(F->part);
  if (F->copy) cudaStreamDestroy(F->copy);
  delete F;
  d->frames = nullptr;
}

extern "C" {

lbx_status lbx_frame_stats_compute(lbx_domain* d, int subs, lbx_frame_stats* out)
{
  if (!d || !out) return ffail(LBX_ERR_INVALID, "NULL argument");
  if (subs < 0 || subs >= d->p.nsubs) return ffail(LBX_ERR_INVALID, "subs out of range");
  Frames* F = frames_of(d);
  if (lbx_status st = alloc_stats(F)) return st;
  // the scratch slot (entries 4 and 5)
  if (lbx_status st = queue_stats(d, F, subs, F->st_dev + 4)) return st;
  FCK(cudaMemcpyAsync(F->st_host + 4, F->st_dev + 4, sizeof(lbx_frame_stats),
                      cudaMemcpyDeviceToHost, d->stream));
  FCK(cudaStreamSynchronize(d->stream));
  *out = F->st_host[4];
  return LBX_OK;
}

lbx_status lbx_frame_enqueue(lbx_domain* d, int time)
{
  if (!d) return ffail(LBX_ERR_INVALID, "domain is NULL");
  Frames* F = frames_of(d);
  if (F->queued - F->waited >= 2)
    return ffail(LBX_ERR_STATE, "two frames are outstanding: lbx_frame_wait first");
  const size_t bytes = (size_t)d->p.nsubs * (1 + d->D) * d->N * d->real_size;
  if (!F->copy) {
    F->bytes = bytes;
    FCK(cudaStreamCreateWithFlags(&F->copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      FCK(cudaMalloc(&F->snap[k], bytes));
      FCK(cudaEventCreateWithFlags(&F->taken[k], cudaEventDisableTiming));
      FCK(cudaEventCreateWithFlags(&F->landed[k], cudaEventDisableTiming));
    }
    for (int k = 0; k < 3; ++k) FCK(cudaHostAlloc(&F->host[k], bytes, cudaHostAllocDefault));
  }
  if (lbx_status st = alloc_stats(F)) return st;
  const int k = (int)(F->queued & 1);
  const int h = (int)(F->queued % 3);
  // The slot's previous frame (queued - 2) was returned by lbx_frame_wait,
  // which waited for its host copy, so its snapshot is free.  Host buffer h
  // last held frame queued - 3, returned before frame queued - 2 was, and
  // the caller was told that its view ends at the second enqueue after its
  // wait, which this one is at the earliest.
  for (int s = 0; s < d->p.nsubs; ++s)
    if (lbx_status st = queue_stats(d, F, s, F->st_dev + 2 * k + s)) return st;
  FCK(cudaMemcpyAsync(F->snap[k], d->mv, bytes, cudaMemcpyDeviceToDevice, d->stream));
  FCK(cudaEventRecord(F->taken[k], d->stream));
  FCK(cudaStreamWaitEvent(F->copy, F->taken[k], 0));
  FCK(cudaMemcpyAsync(F->host[h], F->snap[k], bytes, cudaMemcpyDeviceToHost, F->copy));
  FCK(cudaMemcpyAsync(F->st_host + 2 * k, F->st_dev + 2 * k, 2 * sizeof(lbx_frame_stats),
                      cudaMemcpyDeviceToHost, F->copy));
  FCK(cudaEventRecord(F->landed[k], F->copy));
  F->time[k] = time;
  F->hslot[k] = h;
  F->queued++;
  return LBX_OK;
}

lbx_status lbx_frame_wait(lbx_domain* d, lbx_frame* out)
{
  if (!d || !out) return ffail(LBX_ERR_INVALID, "NULL argument");
  Frames* F = (Frames*)d->frames;
  if (!F || F->queued == F->waited) return ffail(LBX_ERR_STATE, "no frame is outstanding");
  const int k = (int)(F->waited & 1);
  FCK(cudaEventSynchronize(F->landed[k]));
  std::memset(out, 0, sizeof *out);
  out->time = F->time[k];
  out->nsubs = d->p.nsubs;
  const size_t per = (size_t)(1 + d->D) * d->N * d->real_size;
  for (int s = 0; s < d->p.nsubs; ++s) {
    out->mv[s] = (const char*)F->host[F->hslot[k]] + s * per;
    out->stats[s] = F->st_host[2 * k + s];
  }
  F->waited++;
  return LBX_OK;
}

}  // extern "C"
