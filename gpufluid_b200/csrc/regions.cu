// Particle-count-changing steps beside the substep, on the GPU:
//
// Outflow regions: stream compaction of the particles that leave through
// outflow boxes (solver3d.py:1943-1985 k3_mark_alive_outflows +
// k3_scatter_alive, driven by _apply_outflows_gpu :2659-2730).
//
// Reseeding (reseed.py:161-396, reseed_particles_gpu): the binning ranks each
// particle in its cell by id; k_reseed_mark keeps the first max_per_cell of
// each non-solid cell and k_reseed_counts returns the dense per-cell counts
// from which the host builds the emission list; the survivors are compacted
// by the same three launches as the outflows (gf_compact_alive).  The
// emission list is built on the device too: k_deficit_count sums each block
// of cells' deficits (fluid cells under min_per_cell), k_alive_offsets turns
// the sums into offsets, and k_deficit_emit places each cell's deficit at its
// offset in C order of the cells, the order of the reference's np.argwhere /
// np.repeat; only the jitter (drawn from the host generator, as the reference
// draws it) crosses the bus.
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
  const int32_t *alive_in;  // non-null: keep where nonzero (boxes unused)
  int64_t n;
  int32_t *counts;   // [nb] then offsets [nb] then total [1]
};

__device__ __forceinline__ bool alive_of(const RegionArgs &a, int64_t i) {
  if (a.alive_in) return a.alive_in[i] != 0;
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


// The three compaction launches and the read-back of the new count.
static int compact_run(Ctx *c, RegionArgs &a, int nb, int64_t *n_out, const char *what) {
  cudaStream_t st = c->stream;
  int e;
  k_alive_count<<<nb, RG_BLOCK, 0, st>>>(a);
  k_alive_offsets<<<1, RG_BLOCK, 0, st>>>(a.counts, nb);
  k_alive_scatter<<<nb, RG_BLOCK, 0, st>>>(a, nb);
  c->launches += 3;
  if ((e = check_launch(c, what))) return e;
  int32_t total = 0;
  if ((e = check_cuda(c, cudaMemcpyAsync(&total, a.counts + 2 * (int64_t)nb, 4,
                                         cudaMemcpyDeviceToHost, st),
                      "read compacted count")))
    return e;
  if ((e = check_cuda(c, cudaStreamSynchronize(st), "compacted count sync"))) return e;
  *n_out = total;
  return GF_OK;
}

// Block counts [nb], offsets [nb + 1] and `extra` floats, grown on use.
static int region_scratch(Ctx *c, int nb, int64_t extra, int32_t **out) {
  const int64_t need = 2 * (int64_t)nb + 1 + extra;
  if (c->region_scratch_n < need) {
    if (c->region_scratch) cudaFree(c->region_scratch);
    c->region_scratch = nullptr;
    c->region_scratch_n = 0;
    int e = check_cuda(c, cudaMalloc(&c->region_scratch, need * 4), "alloc compaction scratch");
    if (e) return e;
    c->region_scratch_n = need;
  }
  *out = c->region_scratch;
  return GF_OK;
}

// Reseed culling (k_count_particles_per_cell + k_mark_keep_by_rank,
// reseed.py:161-222) on the binned particles: sorted position q holds
// storage slot order[q] with cell key key[slot]; its rank in the cell is
// q - start[key], the binning's canonical order being the particles' ids.
// alive is written by id (original order).
__global__ void k_reseed_mark(const int32_t *__restrict__ order, const int32_t *__restrict__ key,
                              const int32_t *__restrict__ start, const int32_t *__restrict__ pid,
                              const uint8_t *__restrict__ label, int64_t n, int max_per_cell,
                              int ny, int nz, int nty, int ntz, int32_t *__restrict__ alive) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int slot = order[q];
  const int k = key[slot];
  const int rank = (int)(q - start[k]);
  const int t = k >> 9, l = k & 511;
  const int ti = t / (nty * ntz), tj = (t / ntz) % nty, tk = t % ntz;
  const int64_t cell = ((int64_t)(ti * 8 + (l >> 6)) * ny + (tj * 8 + ((l >> 3) & 7))) * nz +
                       (tk * 8 + (l & 7));
  alive[pid[slot]] = (label[cell] != 2 && rank < max_per_cell) ? 1 : 0;
}

// Particles per cell, dense C order, from the binning's per-key counts.
__global__ void k_reseed_counts(const int32_t *__restrict__ count, int nx, int ny, int nz,
                                int nty, int ntz, int32_t *__restrict__ dense) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz) return;
  const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((int64_t)ny * nz));
  const int t = ((i >> 3) * nty + (j >> 3)) * ntz + (k >> 3);
  dense[c] = count[t * 512 + ((i & 7) * 8 + (j & 7)) * 8 + (k & 7)];
}

// Deficit of one cell (reseed.py:345-352): fluid = (marked fluid or holding
// particles) and not solid; deficit = max(min_per_cell - count, 0) there.
__device__ __forceinline__ int deficit_of(uint8_t lab, int cnt, int mn) {
  const bool fluid = (lab == 1 || cnt > 0) && lab != 2;
  return fluid ? max(mn - cnt, 0) : 0;
}

__global__ void __launch_bounds__(RG_BLOCK) k_deficit_count(const uint8_t *__restrict__ label,
                                                            const int32_t *__restrict__ counts,
                                                            int64_t ncell, int mn, int32_t *bsum) {
  __shared__ int ws[RG_BLOCK / 32];
  const int64_t c = blockIdx.x * (int64_t)RG_BLOCK + threadIdx.x;
  int d = c < ncell ? deficit_of(label[c], counts[c], mn) : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = d;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < RG_BLOCK / 32; ++w) t += ws[w];
    bsum[blockIdx.x] = t;
  }
}

// Emitted positions (cell + 0.5 + jitter) * dx, float32 adds in that order.
__global__ void __launch_bounds__(RG_BLOCK) k_deficit_emit(
    const uint8_t *__restrict__ label, const int32_t *__restrict__ counts, int nx, int ny, int nz,
    int mn, const int32_t *__restrict__ boff, const float *__restrict__ jit, float dx,
    float *__restrict__ pos_out) {
  __shared__ int ws[RG_BLOCK / 32];
  const int64_t ncell = (int64_t)nx * ny * nz;
  const int64_t c = blockIdx.x * (int64_t)RG_BLOCK + threadIdx.x;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int d = c < ncell ? deficit_of(label[c], counts[c], mn) : 0;
  int incl = d;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < wid; ++w) before += ws[w];
  if (d == 0) return;
  const int64_t e0 = (int64_t)boff[blockIdx.x] + before + incl - d;
  const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((int64_t)ny * nz));
  const float ci[3] = {__fadd_rn((float)i, 0.5f), __fadd_rn((float)j, 0.5f),
                       __fadd_rn((float)k, 0.5f)};
  for (int r = 0; r < d; ++r) {
    const int64_t e = e0 + r;
#pragma unroll
    for (int a = 0; a < 3; ++a) pos_out[3 * e + a] = __fmul_rn(__fadd_rn(ci[a], jit[3 * e + a]), dx);
  }
}

// Deficit sums and offsets (two launches); the total stays at scratch[2 nb].
static int deficit_offsets(Ctx *c, const uint8_t *label, const int32_t *counts, int mn,
                           int32_t **scratch, int *nb_out) {
  const int nb = (int)((c->ncell + RG_BLOCK - 1) / RG_BLOCK);
  int e = region_scratch(c, nb, 0, scratch);
  if (e) return e;
  k_deficit_count<<<nb, RG_BLOCK, 0, c->stream>>>(label, counts, c->ncell, mn, *scratch);
  k_alive_offsets<<<1, RG_BLOCK, 0, c->stream>>>(*scratch, nb);
  c->launches += 2;
  *nb_out = nb;
  return check_launch(c, "reseed deficit offsets");
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
  if (n == 0) {
    *n_out = 0;
    return GF_OK;
  }
  const int nb = (int)((n + gf::RG_BLOCK - 1) / gf::RG_BLOCK);
  int32_t *counts = nullptr;
  int e = gf::region_scratch(c, nb, 6 * (int64_t)(nbox > 0 ? nbox : 1), &counts);
  if (e) return e;
  float *dbox = reinterpret_cast<float *>(counts + 2 * (int64_t)nb + 1);
  if (nbox > 0 &&
      (e = gf::check_cuda(c, cudaMemcpyAsync(dbox, boxes, (size_t)nbox * 6 * 4,
                                             cudaMemcpyHostToDevice, c->stream),
                          "copy outflow boxes")))
    return e;
  gf::RegionArgs a{pos, vel, pos_out, vel_out, dbox, nbox, nullptr, n, counts};
  return gf::compact_run(c, a, nb, n_out, "gf_outflow_compact");
}

int gf_compact_alive(void *ctx, const float *pos, const float *vel, int64_t n,
                     const int32_t *alive, float *pos_out, float *vel_out, int64_t *n_out) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !n_out || n < 0 || (n > 0 && (!pos || !vel || !alive || !pos_out || !vel_out)))
    return GF_INVALID_ARG;
  if (n > INT32_MAX)
    return gf::fail(c, GF_INVALID_ARG, "gf_compact_alive: particle count exceeds int32 range");
  if (n == 0) {
    *n_out = 0;
    return GF_OK;
  }
  const int nb = (int)((n + gf::RG_BLOCK - 1) / gf::RG_BLOCK);
  int32_t *counts = nullptr;
  int e = gf::region_scratch(c, nb, 0, &counts);
  if (e) return e;
  gf::RegionArgs a{pos, vel, pos_out, vel_out, nullptr, 0, alive, n, counts};
  return gf::compact_run(c, a, nb, n_out, "gf_compact_alive");
}

int gf_reseed_mark(void *ctx, int32_t max_per_cell, int32_t *alive, int32_t *counts) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !counts || max_per_cell < 0 || (c->p.n > 0 && !alive)) return GF_INVALID_ARG;
  if (!c->bound) return gf::fail(c, GF_INVALID_ARG, "gf_reseed_mark: buffers not bound");
  if (c->nseg > 0) return gf::fail(c, GF_INVALID_ARG, "gf_reseed_mark: single-grid contexts only");
  int e = gf::launch_bin(c, GF_FLIP);
  if (e) return e;
  cudaStream_t st = c->stream;
  const int64_t n = c->p.n;
  if (n > 0) {
    gf::k_reseed_mark<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        c->order, c->key, c->start, c->p.pid, c->f.label, n, max_per_cell, c->ny, c->nz,
        c->nty, c->ntz, alive);
    c->launches++;
  }
  gf::k_reseed_counts<<<(unsigned)((c->ncell + 255) / 256), 256, 0, st>>>(
      c->count, c->nx, c->ny, c->nz, c->nty, c->ntz, counts);
  c->launches++;
  return gf::check_launch(c, "gf_reseed_mark");
}

int gf_reseed_deficit(void *ctx, const uint8_t *label, const int32_t *counts,
                      int32_t min_per_cell, int64_t *n_emit) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !label || !counts || !n_emit || min_per_cell < 0) return GF_INVALID_ARG;
  int32_t *scr = nullptr;
  int nb = 0;
  int e = gf::deficit_offsets(c, label, counts, min_per_cell, &scr, &nb);
  if (e) return e;
  int32_t total = 0;
  if ((e = gf::check_cuda(c, cudaMemcpyAsync(&total, scr + 2 * (int64_t)nb, 4,
                                             cudaMemcpyDeviceToHost, c->stream),
                          "read reseed deficit")))
    return e;
  if ((e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "reseed deficit sync"))) return e;
  *n_emit = total;
  return GF_OK;
}

int gf_reseed_emit(void *ctx, const uint8_t *label, const int32_t *counts, int32_t min_per_cell,
                   const float *jitter, float *pos_out) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !label || !counts || !jitter || !pos_out || min_per_cell < 0) return GF_INVALID_ARG;
  int32_t *scr = nullptr;
  int nb = 0;
  int e = gf::deficit_offsets(c, label, counts, min_per_cell, &scr, &nb);
  if (e) return e;
  gf::k_deficit_emit<<<nb, gf::RG_BLOCK, 0, c->stream>>>(label, counts, c->nx, c->ny, c->nz,
                                                         min_per_cell, scr + nb, jitter, c->dx,
                                                         pos_out);
  c->launches++;
  return gf::check_launch(c, "gf_reseed_emit");
}

}  // extern "C"
