// ugks_noalloc.cu -- a block's CFL frequency without any device allocation.
//
// ugks_getDT_noalloc computes what UGKSBlock.getDT obtains from
// ugks_clFindDT + ugks_array_max: the maximum over the interior cells of the
// CFL frequency (dx u + dy v) / A.  The per-cell frequencies are an
// intermediate; where the two-call form keeps them in a caller-provided
// buffer, this entry point keeps them in a fixed array in the library's own
// device memory, so a caller that is not allowed to allocate device memory
// (a host runtime that forbids cudaMalloc inside its time loop, or one that
// drives the solver through a fixed memory plan) can still ask for the time
// step.  The caller passes the inputs and the one-double output only.
#include <cuda_runtime.h>

#include <mutex>

#include "ugks_device.cuh"

using namespace ugks;

// UGKS_NOALLOC_MAX_CELLS (include/ugks_b200.h) interior cells per call: an
// 8 MiB array that every GPU which loads the library holds until exit.
static __device__ __align__(256) double g_cell_frequency[UGKS_NOALLOC_MAX_CELLS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lock;
double *g_scratch[kMaxDevices] = {nullptr};

// device address of the scratch array for the current device, looked up once
int scratch_for_current_device(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return -(int)e;
  if (dev < 0 || dev >= kMaxDevices) return -(int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> guard(g_lock);
  if (g_scratch[dev] == nullptr) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_cell_frequency);
    if (e != cudaSuccess) return -(int)e;
    g_scratch[dev] = static_cast<double *>(p);
  }
  *out = g_scratch[dev];
  return 0;
}

// clFindDT (clKernel.c:224-308) for one cell per thread
__global__ void cell_frequency(ugks_block_desc d, const double *xy, const double *area,
                               const double *macro, double Kn, double *freq) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t n = (size_t)d.ni * d.nj;
  if (t >= n) return;
  const long mi = t / d.nj, mj = t % d.nj;
  freq[t] = cfl_frequency(d, xy, area, ld4(macro, t), mi, mj, Kn);
}

// maximum of freq[0..n) into out[0], one CTA
__global__ void frequency_max(const double *freq, size_t n, double *out) {
  __shared__ double sm[32];
  double m = -INFINITY;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, freq[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = sm[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sm[w]);
    out[0] = r;
  }
}

}  // namespace

extern "C" int ugks_getDT_noalloc(const ugks_block_desc *d, const double *xy, const double *area,
                                  const double *macro, double Kn, double *max_freq, void *stream) {
  const long long n = (long long)d->ni * (long long)d->nj;
  if (d->ni <= 0 || d->nj <= 0) return UGKS_ERR_BAD_SIZE;
  if (n > UGKS_NOALLOC_MAX_CELLS) return UGKS_ERR_TOO_LARGE;
  double *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != 0) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cell_frequency<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(*d, xy, area, macro, Kn, scratch);
  frequency_max<<<1, 1024, 0, st>>>(scratch, (size_t)n, max_freq);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}
