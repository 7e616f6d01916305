// gf_jacobi_noalloc: a Jacobi pressure solve that allocates no device memory.
//
// Some callers cannot allocate GPU memory at the moment they need a pressure
// solve: a host application that owns every device allocation through its
// own pool (a DCC plugin host, a game engine) and forbids libraries from
// calling cudaMalloc or cudaFree behind its back.  They still own the inputs
// and the output; this entry point keeps its only scratch -- the second
// Jacobi buffer -- in a file-scope static device array, so it never calls
// cudaMalloc, cudaFree or any allocating library routine.
//
// The array holds GF_NOALLOC_MAX_CELLS floats (8 MiB).  Every GPU that loads
// the library keeps it until the process exits.  Larger grids are rejected
// with GF_INVALID_ARG.  All calls share the array, so calls that overlap on
// the GPU (different streams, different host threads on the same device)
// race with each other; calls issued in order on one stream are safe.  Each
// call zeroes the part of the array it uses and the output before sweeping.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress while that device is current (host code may not use
// the array's name as a device pointer); make that first call before any
// stream capture begins -- a first call on a capturing stream is refused.
// The label, div and p buffers and the stream must belong to the current
// device.  Errors left pending by earlier, unrelated work on the thread are
// cleared on entry, so the returned status describes this call only.
#include <mutex>

#include "gf_internal.cuh"

namespace gf {

static __device__ __align__(256) float g_jacobi_scratch[GF_NOALLOC_MAX_CELLS];

// One sweep of k3_jacobi_pressure (src/gpufluid/solvers/solver3d.py:878-938) on
// the dense grid: the same neighbour order and float32 operations as the
// compact-tile sweep used by gf_pressure(GF_JACOBI).
__global__ void k_jacobi_dense(const uint8_t *__restrict__ label, const float *__restrict__ div,
                               const float *__restrict__ pin, float *__restrict__ pout, int nx,
                               int ny, int nz) {
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (label[c] != 1) {
      pout[c] = 0.0f;
      continue;
    }
    const int k = (int)(c % nz);
    const int64_t rr = c / nz;
    const int j = (int)(rr % ny), i = (int)(rr / ny);
    const int64_t sx = (int64_t)ny * nz;
    float sum = 0.0f, diag = 0.0f;
    int m;
    if (i > 0) { m = label[c - sx]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c - sx]; } }
    if (i < nx - 1) { m = label[c + sx]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c + sx]; } }
    if (j > 0) { m = label[c - nz]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c - nz]; } }
    if (j < ny - 1) { m = label[c + nz]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c + nz]; } }
    if (k > 0) { m = label[c - 1]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c - 1]; } }
    if (k < nz - 1) { m = label[c + 1]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + pin[c + 1]; } }
    pout[c] = diag < 0.5f ? 0.0f : (sum - div[c]) / diag;
  }
}

// Device address of g_jacobi_scratch per device, looked up once per device
// (refused while `st` is capturing: the lookup must not enter a capture).
static float *scratch_for_current_device(cudaStream_t st, int *status) {
  constexpr int MAX_DEVICES = 64;
  static std::mutex mu;
  static float *addr[MAX_DEVICES] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
    cudaGetLastError();
    *status = GF_NO_DEVICE;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
      cudaGetLastError();
      *status = GF_INVALID_ARG;
      return nullptr;
    }
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_jacobi_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      *status = GF_CUDA_ERROR;
      return nullptr;
    }
    addr[dev] = static_cast<float *>(p);
  }
  *status = GF_OK;
  return addr[dev];
}

}  // namespace gf

extern "C" int gf_jacobi_noalloc(int32_t nx, int32_t ny, int32_t nz, const uint8_t *label,
                                 const float *div, float *p, int32_t iters, void *cuda_stream) {
  if (nx < 1 || ny < 1 || nz < 1 || iters < 0 || !label || !div || !p) return GF_INVALID_ARG;
  const int64_t n = (int64_t)nx * ny * nz;
  if (n > GF_NOALLOC_MAX_CELLS) return GF_INVALID_ARG;  // beyond the static scratch
  cudaGetLastError();  // errors pending from earlier work are not this call's
  cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
  int status = GF_OK;
  float *scratch = gf::scratch_for_current_device(st, &status);
  if (!scratch) return status;
  // the reference starts both Jacobi buffers at zero (solver3d.py:3595)
  if (cudaMemsetAsync(p, 0, n * sizeof(float), st) != cudaSuccess ||
      cudaMemsetAsync(scratch, 0, n * sizeof(float), st) != cudaSuccess) {
    cudaGetLastError();
    return GF_CUDA_ERROR;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t g = (n + 255) / 256;
  if (g > (int64_t)sms * 8) g = (int64_t)sms * 8;
  float *a = p, *b = scratch;
  for (int it = 0; it < iters; ++it) {
    gf::k_jacobi_dense<<<(unsigned)g, 256, 0, st>>>(label, div, a, b, nx, ny, nz);
    float *t = a;
    a = b;
    b = t;
  }
  if (a != p &&
      cudaMemcpyAsync(p, a, n * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return GF_CUDA_ERROR;
  }
  return cudaGetLastError() == cudaSuccess ? GF_OK : GF_CUDA_ERROR;
}
