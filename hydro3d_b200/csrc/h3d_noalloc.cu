// Residual norms of one block with no device allocation.
//
// Some hosts of this solver cannot allocate device memory themselves: code
// running under a memory pool whose budget was committed at start-up, or an
// embedding (a Fortran time loop under a host framework that owns the device
// heap) that forbids cudaMalloc after initialisation.  h3d_residual_noalloc()
// serves them: it evaluates r = b - A p for one block from device arrays the
// caller already owns, and keeps its per-row partial sums in a fixed array in
// this library's own device memory, so the call allocates and frees nothing.
// It copies its four results to host memory and synchronises the stream it
// was given before it returns.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "h3d_internal.h"

namespace {

// Rows (ny * nz) one call can reduce: one partial quadruple per row, plus the
// final quadruple.  4 * 65536 + 4 doubles = 2 MiB of device memory, held by
// every GPU that loads the library until the process exits.
constexpr int kNoAllocMaxRows = 65536;
static __device__ __align__(256) double g_noalloc_scratch[4 * kNoAllocMaxRows + 4];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
int g_sm_count[kMaxDevices] = {0};

// max(a, |r|) that keeps a NaN once one is seen (fmax would drop it, and a
// non-finite residual would then read as a finite max|r|).
__device__ __forceinline__ double nan_max(double a, double v) { return (v != v || v > a) ? v : a; }

// r = b - A p for the interior cells of one row; same operand order as the
// solver's defect (mgsolver.for:707-714).  One warp per row, fixed lane order.
__global__ void __launch_bounds__(256) k_resid_rows(const double* __restrict__ p, const double* __restrict__ b,
                                                    h3d::BlkLev B, double* __restrict__ scratch) {
  const int lane = threadIdx.x & 31;
  const int nrows = B.ny * B.nz;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrows; row += (gridDim.x * blockDim.x) >> 5) {
    const int y = row % B.ny + 1, z = row / B.ny + 1;
    const long long base = (long long)z * B.sxy + (long long)y * B.sx;
    double rr = 0, bb = 0, rm = 0, rs = 0;
    for (int x = 1 + lane; x <= B.nx; x += 32) {
      const long long i = base + x;
      const int ph = B.phys;
      const double aw = (x == 1 && (ph & 1)) ? 0.0 : B.ax, ae = (x == B.nx && (ph & 2)) ? 0.0 : B.ax;
      const double as = (y == 1 && (ph & 4)) ? 0.0 : B.ay, an = (y == B.ny && (ph & 8)) ? 0.0 : B.ay;
      const double ab = (z == 1 && (ph & 16)) ? 0.0 : B.az, at = (z == B.nz && (ph & 32)) ? 0.0 : B.az;
      const double ap = -(aw + ae + as + an + ab + at);
      const double bv = b[i];
      const double r = bv - (aw * p[i - 1] + ae * p[i + 1] + as * p[i - B.sx] + an * p[i + B.sx] +
                             ab * p[i - B.sxy] + at * p[i + B.sxy] + ap * p[i]);
      rr += r * r;
      bb += bv * bv;
      rm = nan_max(rm, fabs(r) * B.dv);
      rs += r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rr += __shfl_xor_sync(0xffffffffu, rr, o);
      bb += __shfl_xor_sync(0xffffffffu, bb, o);
      rm = nan_max(rm, __shfl_xor_sync(0xffffffffu, rm, o));
      rs += __shfl_xor_sync(0xffffffffu, rs, o);
    }
    if (lane == 0) {
      scratch[4 * (size_t)row + 0] = rr;
      scratch[4 * (size_t)row + 1] = bb;
      scratch[4 * (size_t)row + 2] = rm;
      scratch[4 * (size_t)row + 3] = rs;
    }
  }
}

// Fixed-order reduction of the row partials into scratch[4*nrows .. +3].
__global__ void __launch_bounds__(256) k_resid_reduce(double* __restrict__ scratch, int nrows) {
  __shared__ double sh[4][256];
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (int q = threadIdx.x; q < nrows; q += 256) {
    a0 += scratch[4 * (size_t)q];
    a1 += scratch[4 * (size_t)q + 1];
    a2 = nan_max(a2, scratch[4 * (size_t)q + 2]);
    a3 += scratch[4 * (size_t)q + 3];
  }
  sh[0][threadIdx.x] = a0; sh[1][threadIdx.x] = a1; sh[2][threadIdx.x] = a2; sh[3][threadIdx.x] = a3;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sh[0][threadIdx.x] += sh[0][threadIdx.x + s];
      sh[1][threadIdx.x] += sh[1][threadIdx.x + s];
      sh[2][threadIdx.x] = nan_max(sh[2][threadIdx.x], sh[2][threadIdx.x + s]);
      sh[3][threadIdx.x] += sh[3][threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) scratch[4 * (size_t)nrows + k] = sh[k][0];
}

// Device address of the scratch array on the current device and that
// device's multiprocessor count (set-up, once per device; the array's
// host-side name is only a stand-in for its address).
int scratch_of_current_device(double** out, int* sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    h3d::set_call_error("h3d_residual_noalloc: no current CUDA device");
    return H3D_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    double* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      h3d::set_call_error(std::string("h3d_residual_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return H3D_ERR_CUDA;
    }
    int nsm = 0;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || nsm < 1) {
      h3d::set_call_error(std::string("h3d_residual_noalloc: cudaDeviceGetAttribute: ") + cudaGetErrorString(e));
      return H3D_ERR_CUDA;
    }
    g_sm_count[dev] = nsm;
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  *sms = g_sm_count[dev];
  return H3D_OK;
}

}  // namespace

extern "C" int h3d_residual_noalloc(const double* p, const double* b, int32_t nx, int32_t ny, int32_t nz,
                                    const double* h, int32_t phys_mask, double* out, void* stream) {
  if (!p || !b || !h || !out || nx < 1 || ny < 1 || nz < 1) {
    h3d::set_call_error("h3d_residual_noalloc: null pointer or empty block");
    return H3D_ERR_ARG;
  }
  {
    // it copies to host memory and synchronises the stream: neither may be
    // captured into a graph, so a capturing stream is refused before any work
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs);
    if (e != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      h3d::set_call_error("h3d_residual_noalloc: the stream is being captured into a CUDA graph; this call copies "
                          "its result to host memory and synchronises the stream, so it cannot be captured");
      return H3D_ERR_ARG;
    }
  }
  if ((long long)ny * nz > kNoAllocMaxRows) {
    h3d::set_call_error("h3d_residual_noalloc: block has ny*nz = " + std::to_string((long long)ny * nz) +
                        " rows; the allocation-free residual handles at most " + std::to_string(kNoAllocMaxRows));
    return H3D_ERR_ARG;
  }
  double* scratch = nullptr;
  int sms = 0;
  int rc = scratch_of_current_device(&scratch, &sms);
  if (rc != H3D_OK) return rc;
  h3d::BlkLev B{};
  B.nx = nx; B.ny = ny; B.nz = nz;
  B.sx = nx + 2;
  B.sxy = (long long)(nx + 2) * (ny + 2);
  B.off = 0;
  B.phys = phys_mask & 63;
  B.ax = 1.0 / (h[0] * h[0]);
  B.ay = 1.0 / (h[1] * h[1]);
  B.az = 1.0 / (h[2] * h[2]);
  B.dv = h[0] * h[1] * h[2];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nrows = ny * nz;
  int grid = (nrows + 7) / 8;
  if (grid > sms * 8) grid = sms * 8;
  k_resid_rows<<<grid, 256, 0, st>>>(p, b, B, scratch);
  k_resid_reduce<<<1, 256, 0, st>>>(scratch, nrows);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch + 4 * (size_t)nrows, 4 * sizeof(double),
                                            cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    h3d::set_call_error(std::string("h3d_residual_noalloc: ") + cudaGetErrorString(e));
    return H3D_ERR_CUDA;
  }
  return H3D_OK;
}
