// Particle binning for one substep.
//
// Replaces the cell/label part of k3_p2g (src/gpufluid/solvers/solver3d.py:
// 92-101) and adds what the reference does not have: a canonical sort of the
// particles by (tile-major cell key, original particle id), so that P2G can
// work tile by tile out of shared memory and G2P reads particles coalesced.
//
//   k_clear_labels  label <- 2 if solid else 0        (k3_clear_grid :62-65)
//   k_bin_keys      cell = clamp(int(p/dx)), label 1 unless solid, key,
//                   per-key count with warp-aggregated atomics
//   k_scan_*        exclusive scan of the per-key counts -> start
//   k_place         slot = start[key] + rank
//   k_canon         order each cell's segment by particle id (rank by count)
//   k_permute       gather caller AoS buffers into sorted float4 records
#include "gf_internal.cuh"

namespace gf {

__global__ void k_clear_labels(uint8_t *__restrict__ label, int64_t n) {
  // byte values are 0/1/2: keeping only bit 1 maps 2->2 and 0,1->0
  int64_t nw = n >> 2;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  uint32_t *w = reinterpret_cast<uint32_t *>(label);
  for (int64_t q = i; q < nw; q += stride) w[q] &= 0x02020202u;
  for (int64_t q = (nw << 2) + i; q < n; q += stride) label[q] &= 0x02u;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

__global__ void k_bin_keys(const float *__restrict__ pos, int64_t n, float dx, float inv, int nx,
                           int ny, int nz, int nty, int ntz, uint8_t *__restrict__ label,
                           int32_t *__restrict__ key, int32_t *__restrict__ rank,
                           int32_t *__restrict__ count, int64_t nkeys) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned amask = __ballot_sync(0xffffffffu, i < n);
  if (i >= n) return;
  float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
  // int(p / dx) with IEEE division (a product when dx is a power of two) and
  // truncation toward zero, then clamped
  int ci = clampi(__float2int_rz(div_dx(px, dx, inv)), 0, nx - 1);
  int cj = clampi(__float2int_rz(div_dx(py, dx, inv)), 0, ny - 1);
  int ck = clampi(__float2int_rz(div_dx(pz, dx, inv)), 0, nz - 1);
  int64_t cell = ((int64_t)ci * ny + cj) * nz + ck;
  if (GF_IN(cell, (int64_t)nx * ny * nz) && label[cell] != 2)
    label[cell] = 1;  // benign race: every writer stores 1
  int t = ((ci >> 3) * nty + (cj >> 3)) * ntz + (ck >> 3);
  int kk = t * TILE_CELLS + (((ci & 7) * 8 + (cj & 7)) * 8 + (ck & 7));
  key[i] = kk;
  unsigned lane = threadIdx.x & 31u;
  unsigned peers = __match_any_sync(amask, kk);
  int leader = __ffs(peers) - 1;
  int below = __popc(peers & ((1u << lane) - 1u));
  int base = 0;
  if ((int)lane == leader && GF_IN(kk, nkeys)) base = atomicAdd(&count[kk], __popc(peers));
  base = __shfl_sync(amask, base, leader);
  rank[i] = base + below;
}

// k_bin_keys over a batch: each particle finds its scene in the particle
// prefix of the segment table and bins into that scene's cells and tiles.
__global__ void kb_bin_keys(const float *__restrict__ pos, int64_t n, SegIndex sx,
                            uint8_t *__restrict__ label, int32_t *__restrict__ key,
                            int32_t *__restrict__ rank, int32_t *__restrict__ count,
                            int64_t ncell, int64_t nkeys) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned amask = __ballot_sync(0xffffffffu, i < n);
  if (i >= n) return;
  const SegRow r = sx.row[seg_find(sx.part0, sx.n, i)];
  float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
  int ci = clampi(__float2int_rz(__fdiv_rn(px, r.dx)), 0, r.nx - 1);
  int cj = clampi(__float2int_rz(__fdiv_rn(py, r.dx)), 0, r.ny - 1);
  int ck = clampi(__float2int_rz(__fdiv_rn(pz, r.dx)), 0, r.nz - 1);
  int64_t cell = r.cell0 + ((int64_t)ci * r.ny + cj) * r.nz + ck;
  if (GF_IN(cell, ncell) && label[cell] != 2) label[cell] = 1;
  int64_t t = r.tile0 + ((ci >> 3) * r.nty + (cj >> 3)) * r.ntz + (ck >> 3);
  int kk = (int)(t * TILE_CELLS + (((ci & 7) * 8 + (cj & 7)) * 8 + (ck & 7)));
  key[i] = kk;
  unsigned lane = threadIdx.x & 31u;
  unsigned peers = __match_any_sync(amask, kk);
  int leader = __ffs(peers) - 1;
  int below = __popc(peers & ((1u << lane) - 1u));
  int base = 0;
  if ((int)lane == leader && GF_IN(kk, nkeys)) base = atomicAdd(&count[kk], __popc(peers));
  base = __shfl_sync(amask, base, leader);
  rank[i] = base + below;
}

// ---- exclusive scan of int32 counts (3 kernels, 4096 elements per block) ----
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int warp_incl_scan(int v) {
  unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (unsigned)o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread (blockDim.x <= 1024).
__device__ int block_excl_scan(int v) {
  __shared__ int warp_sums[32];
  unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  unsigned nw = blockDim.x >> 5;
  int incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int s = lane < nw ? warp_sums[lane] : 0;
    int si = warp_incl_scan(s);
    if (lane < nw) warp_sums[lane] = si - s;
  }
  __syncthreads();
  int res = warp_sums[wid] + incl - v;
  __syncthreads();  // warp_sums may be rewritten by the next call
  return res;
}

__global__ void k_scan_block_sums(const int32_t *__restrict__ cnt, int64_t n,
                                  int32_t *__restrict__ part) {
  int64_t base = blockIdx.x * (int64_t)SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
  int s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q)
    if (base + q < n) s += cnt[base + q];
  // block reduction
  __shared__ int red[SCAN_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
  }
}

// Exclusive scan of the block sums in place (one block, nb <= SCAN_CHUNK).
__global__ void k_scan_parts(int32_t *__restrict__ part, int64_t nb, int32_t *__restrict__ total) {
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t off = 0; off < nb; off += SCAN_CHUNK) {
    int64_t base = off + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
      v[q] = base + q < nb ? part[base + q] : 0;
      s += v[q];
    }
    int pre = block_excl_scan(s);
    __shared__ int blk_total;
    if (threadIdx.x == blockDim.x - 1) blk_total = pre + s;
    __syncthreads();
    int run = carry + pre;
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
      if (base + q < nb) part[base + q] = run;
      run += v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += blk_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_final(const int32_t *__restrict__ cnt, int64_t n,
                             const int32_t *__restrict__ part, int32_t *__restrict__ start,
                             const int32_t *__restrict__ total) {
  int64_t base = blockIdx.x * (int64_t)SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
  int v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    v[q] = base + q < n ? cnt[base + q] : 0;
    s += v[q];
  }
  int run = part[blockIdx.x] + block_excl_scan(s);
#pragma unroll
  for (int q = 0; q < SCAN_ITEMS; ++q) {
    if (base + q < n) start[base + q] = run;
    run += v[q];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) start[n] = *total;
}

__global__ void k_place(const int32_t *__restrict__ key, const int32_t *__restrict__ rank,
                        const int32_t *__restrict__ start, int64_t n,
                        int32_t *__restrict__ order) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t slot = (int64_t)start[key[i]] + rank[i];
  if (GF_IN(slot, n)) order[slot] = (int32_t)i;
}

// Canonical order of each cell segment, by original particle id: slot d of
// the placement order (k_place, whose order within a cell follows the
// atomics) moves to s + the number of its cell's particles with a smaller id
// (ties, which unique ids never have, broken by index, so the result is a
// permutation whatever the ids).  One thread per slot; its cell's ids are read
// through the placement order, so a cell of c particles costs c^2 compares
// spread over c threads.  The result goes to `canon` (the rank array, dead
// after k_place).
__global__ void k_canon(const int32_t *__restrict__ key, const int32_t *__restrict__ count,
                        const int32_t *__restrict__ start, const int32_t *__restrict__ pid,
                        const int32_t *__restrict__ order, int32_t *__restrict__ canon,
                        int64_t n, int64_t nkeys) {
  const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (d >= n) return;
  const int32_t i = order[d];
  if (!GF_IN(i, n)) return;
  const int32_t k = key[i];
  if (!GF_IN(k, nkeys)) return;
  const int32_t s = start[k], cnt = count[k];
  if (!GF_IN(s, n) || !GF_IN((int64_t)s + cnt - 1, n)) return;
  const int32_t id = pid[i];
  int32_t r = 0;
  for (int32_t a = 0; a < cnt; ++a) {
    const int32_t j = order[s + a];
    const int32_t pj = pid[j];
    r += (pj < id || (pj == id && j < i)) ? 1 : 0;
  }
  canon[s + r] = i;
}

// Sorted float4 records of the canonical order (canon), which also becomes
// the context's order array for the later stages.
__global__ void k_permute(const int32_t *__restrict__ canon, int64_t n,
                          const float *__restrict__ pos, const float *__restrict__ vel,
                          const float *__restrict__ C, const int32_t *__restrict__ pid,
                          float4 *__restrict__ rec0, float4 *__restrict__ rec1,
                          float4 *__restrict__ rec2, float4 *__restrict__ rec3,
                          int32_t *__restrict__ order) {
  int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (d >= n) return;
  int64_t s = canon[d];
  order[d] = (int32_t)s;
  if (!GF_IN(s, n)) return;
  float4 a, b;
  a.x = pos[3 * s];
  a.y = pos[3 * s + 1];
  a.z = pos[3 * s + 2];
  a.w = __int_as_float(pid[s]);
  b.x = vel[3 * s];
  b.y = vel[3 * s + 1];
  b.z = vel[3 * s + 2];
  b.w = 0.f;
  if (C) {  // APIC: one record per face component c, (v_c, C row c)
    const float *m = C + 9 * s;
    rec2[d] = make_float4(b.y, m[3], m[4], m[5]);
    rec3[d] = make_float4(b.z, m[6], m[7], m[8]);
    b = make_float4(b.x, m[0], m[1], m[2]);
  }
  rec0[d] = a;
  rec1[d] = b;
}

static inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int launch_bin(Ctx *c, int transfer) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_bin: buffers not bound");
  const int64_t n = c->p.n;
  cudaStream_t st = c->stream;
  int e;
  {
    int64_t nw = c->ncell >> 2;
    unsigned g = nblk(nw > 0 ? nw : 1, 256);
    if (g > 4096) g = 4096;
    k_clear_labels<<<g, 256, 0, st>>>(c->f.label, c->ncell);
    c->launches++;
  }
  if ((e = check_cuda(c, cudaMemsetAsync(c->count, 0, c->nkeys * sizeof(int32_t), st),
                      "memset count")))
    return e;
  if (n > 0 && c->nseg > 0) {
    kb_bin_keys<<<nblk(n, 256), 256, 0, st>>>(c->p.pos, n, seg_index(c), c->f.label, c->key,
                                              c->rank, c->count, c->ncell, c->nkeys);
    c->launches++;
  } else if (n > 0) {
    k_bin_keys<<<nblk(n, 256), 256, 0, st>>>(c->p.pos, n, c->dx, exact_inverse(c->dx), c->nx,
                                             c->ny, c->nz,
                                             c->nty, c->ntz, c->f.label, c->key, c->rank,
                                             c->count, c->nkeys);
    c->launches++;
  }
  k_scan_block_sums<<<(unsigned)c->n_scan_blocks, SCAN_THREADS, 0, st>>>(c->count, c->nkeys,
                                                                        c->scan_part);
  k_scan_parts<<<1, SCAN_THREADS, 0, st>>>(c->scan_part, c->n_scan_blocks,
                                           c->scan_part + c->n_scan_blocks);
  k_scan_final<<<(unsigned)c->n_scan_blocks, SCAN_THREADS, 0, st>>>(
      c->count, c->nkeys, c->scan_part, c->start, c->scan_part + c->n_scan_blocks);
  c->launches += 3;
  if (n > 0) {
    k_place<<<nblk(n, 256), 256, 0, st>>>(c->key, c->rank, c->start, n, c->order);
    k_canon<<<nblk(n, 256), 256, 0, st>>>(c->key, c->count, c->start, c->p.pid, c->order,
                                          c->rank, n, c->nkeys);
    const float *Cp = transfer == GF_APIC ? c->p.C : nullptr;
    k_permute<<<nblk(n, 256), 256, 0, st>>>(c->rank, n, c->p.pos, c->p.vel, Cp, c->p.pid,
                                            c->rec0, c->rec1, c->rec2, c->rec3, c->order);
    c->launches += 3;
  }
  return check_launch(c, "gf_bin");
}

GF_BOUNDS_READER(bin)

}  // namespace gf
