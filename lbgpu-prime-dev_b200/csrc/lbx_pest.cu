// lbx_pest.cu -- PEST point sampling (PEST_OUTPUT_ON).
//
// The reference keeps a time-ordered list of (time, x, y) samples
// (read_PEST_in_files, src/latman.c:899-1046).  Before each step whose time
// is the next sample's, it sets pest_output_flag_c so the kernel writes the
// flow's u and the solute's C (src/k_stream_collide_stream.c:297-324,
// PEST_gpu_switch, src/latman.c:1048-1065); after the step it copies C, u_x
// and u_y of each due sample's node to the host, three synchronous 1-value
// cudaMemcpy calls per sample (write_PEST_out_data, src/latman.c:1067-1176).
// Here the step writes the macro variables and one small gather kernel puts
// every due sample's values into a device array, read once at the end.
#include "lbx.h"
#include "lbx_internal.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <vector>

namespace {

lbx_status pfail(lbx_status code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));

lbx_status pfail(lbx_status code, const char* fmt, ...)
{
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return lbx_internal_fail(code, buf);
}

#define PCK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return pfail(e_ == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA,        \
                   "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

struct Pest {
  std::vector<int> time, node;   // kept samples, in order
  int* node_dev = nullptr;       // [count]
  void* vals = nullptr;          // [count][3] reals: C, u_x, u_y
  int cursor = 0;                // samples taken so far
};

// vals[k] = (C of the solute, u_x and u_y of the flow) at node[k], for the
// samples k in [first, first + cnt).
template <typename T>
__global__ void pest_gather(const T* __restrict__ mv, long long N, int D,
                            const int* __restrict__ node, int first, int cnt, T* __restrict__ vals)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int k = first + i;
  const long long n = node[k];
  const T* flow = mv;
  const T* solute = mv + (long long)(1 + D) * N;
  vals[3 * k + 0] = solute[n];
  vals[3 * k + 1] = flow[N + n];
  vals[3 * k + 2] = flow[2 * N + n];
}

void pest_release(Pest* P)
{
  cudaFree(P->node_dev);
  cudaFree(P->vals);
  delete P;
}

}  // namespace

bool lbx_internal_pest_due(const lbx_domain* d, int t)
{
  const Pest* P = (const Pest*)d->pest;
  return P && P->cursor < (int)P->time.size() && P->time[P->cursor] == t;
}

lbx_status lbx_internal_pest_after(lbx_domain* d, int t)
{
  Pest* P = (Pest*)d->pest;
  if (!lbx_internal_pest_due(d, t)) return LBX_OK;
  const int first = P->cursor;
  int k = first;
  while (k < (int)P->time.size() && P->time[k] == t) ++k;
  const int cnt = k - first;
  const unsigned blocks = (unsigned)((cnt + 127) / 128);
  if (d->real_size == 8)
    pest_gather<double><<<blocks, 128, 0, d->stream>>>((const double*)d->mv, d->N, d->D,
                                                        P->node_dev, first, cnt, (double*)P->vals);
  else
    pest_gather<float><<<blocks, 128, 0, d->stream>>>((const float*)d->mv, d->N, d->D,
                                                      P->node_dev, first, cnt, (float*)P->vals);
  d->launches++;
  PCK(cudaGetLastError());
  P->cursor = k;
  return LBX_OK;
}

void lbx_internal_pest_free(lbx_domain* d)
{
  if (d->pest) pest_release((Pest*)d->pest);
  d->pest = nullptr;
}

extern "C" {

lbx_status lbx_pest_set(lbx_domain* d, int count, const int* time, const int* node)
{
  if (!d) return pfail(LBX_ERR_INVALID, "domain is NULL");
  if (count < 0 || (count > 0 && (!time || !node)))
    return pfail(LBX_ERR_INVALID, "need count >= 0 and the time and node arrays");
  if (count > 0 && d->p.nsubs != 2)
    return pfail(LBX_ERR_INVALID, "PEST samples read the solute: nsubs must be 2");
  for (int k = 0; k < count; ++k) {
    if (node[k] < 0 || node[k] >= d->N)
      return pfail(LBX_ERR_INVALID, "sample %d: node %d outside the lattice", k, node[k]);
    if (k > 0 && time[k] < time[k - 1])
      return pfail(LBX_ERR_INVALID, "sample %d: times must not decrease", k);
  }
  PCK(cudaStreamSynchronize(d->stream));
  lbx_internal_pest_free(d);
  if (count == 0) return LBX_OK;
  Pest* P = new Pest();
  P->time.assign(time, time + count);
  P->node.assign(node, node + count);
  cudaError_t e = cudaMalloc(&P->node_dev, (size_t)count * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&P->vals, (size_t)count * 3 * d->real_size);
  if (e == cudaSuccess)
    e = cudaMemcpy(P->node_dev, node, (size_t)count * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(P->vals, 0, (size_t)count * 3 * d->real_size);
  if (e != cudaSuccess) {
    pest_release(P);
    return pfail(e == cudaErrorMemoryAllocation ? LBX_ERR_NOMEM : LBX_ERR_CUDA, "PEST buffers: %s",
                 cudaGetErrorString(e));
  }
  d->pest = P;
  lbx_internal_drop_graphs(d);
  return LBX_OK;
}

lbx_status lbx_pest_read(lbx_domain* d, double* conc, double* ux, double* uy, int* taken)
{
  if (!d) return pfail(LBX_ERR_INVALID, "domain is NULL");
  Pest* P = (Pest*)d->pest;
  const int count = P ? (int)P->time.size() : 0;
  if (taken) *taken = P ? P->cursor : 0;
  if (count == 0) return LBX_OK;
  if (!conc || !ux || !uy) return pfail(LBX_ERR_INVALID, "NULL output array");
  PCK(cudaStreamSynchronize(d->stream));
  std::vector<double> v((size_t)count * 3);
  if (d->real_size == 8) {
    PCK(cudaMemcpy(v.data(), P->vals, v.size() * sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    std::vector<float> h(v.size());
    PCK(cudaMemcpy(h.data(), P->vals, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < h.size(); ++i) v[i] = h[i];
  }
  for (int k = 0; k < count; ++k) {
    const bool got = k < P->cursor;
    conc[k] = got ? v[3 * k] : NAN;
    ux[k] = got ? v[3 * k + 1] : NAN;
    uy[k] = got ? v[3 * k + 2] : NAN;
  }
  return LBX_OK;
}

}  // extern "C"
