// Outflow regions: GPU stream compaction of the particles that leave through
// outflow boxes (solver3d.py:1943-1985 k3_mark_alive_outflows +
// k3_scatter_alive, driven by _apply_outflows_gpu :2659-2730).
//
// A particle is removed when it lies inside ANY box (lo <= p <= hi on all
// three axes, float32 compares); the survivors keep their relative order
// (the reference's inclusive prefix sum: destination = prefix - 1).  Three
// launches over blocks of 1024 particles:
//   k_alive_count    alive flags counted per block (__syncthreads_count)
//   k_alive_offsets  one block turns the per-block counts into exclusive
//                    offsets and the total
//   k_alive_scatter  each survivor's rank inside its block (warp ballots and
//                    a warp-prefix in shared memory) plus its block's offset
// The new count is read back to the host, as the reference reads the last
// prefix value.  Integer and copy work only: the result is bit-exact.
#include "gf_internal.cuh"

namespace gf {

constexpr int RG_BLOCK = 1024;

struct RegionArgs {
  const float *pos, *vel;
  float *pos_out, *vel_out;
  const float *box;  // nbox x (lo.xyz, hi.xyz)
  int nbox;
  int64_t n;
  int32_t *counts;   // [nb] then offsets [nb] then total [1]
};

__device__ __forceinline__ bool alive_of(const RegionArgs &a, int64_t i) {
  const float x = a.pos[3 * i], y = a.pos[3 * i + 1], z = a.pos[3 * i + 2];
  bool alive = true;
  for (int j = 0; j < a.nbox; ++j) {
    const float *b = a.box + 6 * j;
    if (x >= b[0] && x <= b[3] && y >= b[1] && y <= b[4] && z >= b[2] && z <= b[5]) alive = false;
  }
  return alive;
}

__global__ void __launch_bounds__(RG_BLOCK) k_alive_count(RegionArgs a) {
  const int64_t i = blockIdx.x * (int64_t)RG_BLOCK + threadIdx.x;
  const int alive = i < a.n && alive_of(a, i);
  const int cnt = __syncthreads_count(alive);
  if (threadIdx.x == 0) a.counts[blockIdx.x] = cnt;
}

// Exclusive offsets of nb block counts (one block, chunks of 1024).
__global__ void __launch_bounds__(RG_BLOCK) k_alive_offsets(int32_t *counts, int nb) {
  __shared__ int warp_sums[RG_BLOCK / 32];
  __shared__ int carry;
  int32_t *offsets = counts + nb;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += RG_BLOCK) {
    const int t = base + threadIdx.x;
    const int v = t < nb ? counts[t] : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int s = warp_sums[lane];
      int si = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += u;
      }
      warp_sums[lane] = si - s;  // exclusive prefix of the warp sums
    }
    __syncthreads();
    if (t < nb) offsets[t] = carry + warp_sums[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == RG_BLOCK - 1) carry += warp_sums[wid] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) offsets[nb] = carry;  // the new particle count
}

__global__ void __launch_bounds__(RG_BLOCK) k_alive_scatter(RegionArgs a, int nb) {
  __shared__ int warp_cnt[RG_BLOCK / 32];
  const int64_t i = blockIdx.x * (int64_t)RG_BLOCK + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool alive = i < a.n && alive_of(a, i);
  const unsigned ballot = __ballot_sync(0xffffffffu, alive);
  if (lane == 0) warp_cnt[wid] = __popc(ballot);
  __syncthreads();
  int before = 0;
  for (int w = 0; w < wid; ++w) before += warp_cnt[w];
  if (!alive) return;
  const int64_t dst = (int64_t)a.counts[nb + blockIdx.x] + before +
                      __popc(ballot & ((1u << lane) - 1u));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    a.pos_out[3 * dst + d] = a.pos[3 * i + d];
    a.vel_out[3 * dst + d] = a.vel[3 * i + d];
  }
}

}  // namespace gf

using gf::Ctx;

extern "C" {

int gf_outflow_compact(void *ctx, const float *pos, const float *vel, int64_t n,
                       const float *boxes, int32_t nbox, float *pos_out, float *vel_out,
                       int64_t *n_out) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !n_out || n < 0 || nbox < 0 || (nbox > 0 && !boxes) ||
      (n > 0 && (!pos || !vel || !pos_out || !vel_out)))
    return GF_INVALID_ARG;
  if (n > INT32_MAX)
    return gf::fail(c, GF_INVALID_ARG, "gf_outflow_compact: particle count exceeds int32 range");
  for (int32_t j = 0; j < nbox; ++j)
    for (int d = 0; d < 3; ++d)
      if (boxes[6 * j + 3 + d] < boxes[6 * j + d])
        return gf::fail(c, GF_INVALID_ARG, "gf_outflow_compact: a box has hi < lo");
  cudaStream_t st = c->stream;
  int e;
  if (n == 0) {
    *n_out = 0;
    return GF_OK;
  }
  const int nb = (int)((n + gf::RG_BLOCK - 1) / gf::RG_BLOCK);
  // scratch: counts [nb], offsets [nb + 1], then the boxes (6 floats each)
  const int64_t need = 2 * (int64_t)nb + 1 + 6 * (int64_t)(nbox > 0 ? nbox : 1);
  if (c->region_scratch_n < need) {
    if (c->region_scratch) cudaFree(c->region_scratch);
    c->region_scratch = nullptr;
    c->region_scratch_n = 0;
    if ((e = gf::check_cuda(c, cudaMalloc(&c->region_scratch, need * 4), "alloc outflow scratch")))
      return e;
    c->region_scratch_n = need;
  }
  int32_t *counts = c->region_scratch;
  float *dbox = reinterpret_cast<float *>(counts + 2 * (int64_t)nb + 1);
  if (nbox > 0 &&
      (e = gf::check_cuda(c, cudaMemcpyAsync(dbox, boxes, (size_t)nbox * 6 * 4,
                                             cudaMemcpyHostToDevice, st),
                          "copy outflow boxes")))
    return e;
  gf::RegionArgs a{pos, vel, pos_out, vel_out, dbox, nbox, n, counts};
  gf::k_alive_count<<<nb, gf::RG_BLOCK, 0, st>>>(a);
  gf::k_alive_offsets<<<1, gf::RG_BLOCK, 0, st>>>(counts, nb);
  gf::k_alive_scatter<<<nb, gf::RG_BLOCK, 0, st>>>(a, nb);
  c->launches += 3;
  if ((e = gf::check_launch(c, "gf_outflow_compact"))) return e;
  int32_t total = 0;
  if ((e = gf::check_cuda(c, cudaMemcpyAsync(&total, counts + 2 * (int64_t)nb, 4,
                                             cudaMemcpyDeviceToHost, st),
                          "read outflow count")))
    return e;
  if ((e = gf::check_cuda(c, cudaStreamSynchronize(st), "outflow count sync"))) return e;
  *n_out = total;
  return GF_OK;
}

}  // extern "C"
