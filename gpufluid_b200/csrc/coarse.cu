// Set-up of the coarse correction of the pressure PCG (GF_FLAG_COARSE), run
// before each solve.  The preconditioner is additive two-level,
// M^-1 = M_tile^-1 + P B P^T, with P the indicator of the fluid cells of a set
// of regions and B = A_c^-1, A_c = P^T A P (no counterpart in the reference,
// whose solves use the Jacobi preconditioner only):
//   * the shared-memory solver (k_pcg_smem): one region per active 8^3 tile;
//   * the global-memory solver (k_pcg, tile SGS preconditioner): one region
//     per cube of CT^3 tiles (CT = Ctx::rg_ct, the smallest power of two that
//     keeps the region grid within COARSE_RG_DENSE_MAX regions).
// A_c has the 7-point pattern of the region grid: the diagonal of region R is
// the sum over its fluid cells of diag - #fluid neighbours inside R, the entry
// for the neighbouring region across face d is minus the fluid-fluid faces
// across it.  Row R of B solves A_c x = e_R by Jacobi-preconditioned CG in
// float32 to ||e_R - A_c x|| <= 1e-3 (B only has to be close to the inverse
// for the correction to work), warm-started from the last solve's row of the
// same region with its columns mapped by region id; the rows are stored as
// bfloat16 (an FP64 study of the 128^3 bench system needed the same number of
// PCG iterations with B rounded to 7 mantissa bits as with the exact B).
#include <cuda_bf16.h>

#include "gf_internal.cuh"

namespace gf {

constexpr float kCoarseTol2 = 1e-6f;  // squared residual target of the row solves
constexpr int COARSE_SOLVE_THREADS = 256;

__device__ __forceinline__ float bf16_at(const uint16_t *p, int64_t i) {
  return __uint_as_float((unsigned)p[i] << 16);
}

// Whether the set-up of this solve runs: its region count is within the
// buffers and the solver that uses it will run (gate: the shared-memory
// solver deferred to the global one).
__device__ __forceinline__ bool coarse_active(const CoarseSetup &a, int n) {
  return n > 0 && n <= a.limit && n <= COARSE_RMAX && (a.gate == nullptr || *a.gate != 0);
}

// ---- tile regions: row t of A_c for active tile slot t (one block per slot)
__global__ void __launch_bounds__(256) k_coarse_tile_rows(CoarseSetup a,
                                                          const uint16_t *__restrict__ code) {
  const int na = *a.count;
  const int s = blockIdx.x;
  if (!coarse_active(a, na) || s >= na) return;
  float v[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // diagonal, then faces 0..5
  for (int L = threadIdx.x; L < 512; L += blockDim.x) {
    const uint16_t cd = code[(int64_t)s * 512 + L];
    if (!(cd & CODE_FLUID)) continue;
    const int li = L >> 6, lj = (L >> 3) & 7, lk = L & 7;
    int same = 0;
#pragma unroll
    for (int dir = 0; dir < 6; ++dir) {
      if (!(cd & (1 << dir))) continue;
      const bool inside = dir == 0 ? li > 0 : dir == 1 ? li < 7 : dir == 2 ? lj > 0
                        : dir == 3 ? lj < 7 : dir == 4 ? lk > 0 : lk < 7;
      if (inside) ++same; else v[1 + dir] += 1.f;
    }
    v[0] += (float)((int)((cd >> CODE_DIAG_SHIFT) & 7) - same);
  }
  __shared__ float red[8][7];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 7; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0) red[wid][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    if (threadIdx.x == 0) {
      a.cdiag[s] = t > 0.f ? t : 1.0f;  // an empty region decouples
    } else {
      const int dir = threadIdx.x - 1;
      a.coff[(int64_t)s * 6 + dir] = a.nbr[(int64_t)s * 6 + dir] >= 0 ? -t : 0.f;
    }
  }
}

// ---- cube regions of CT^3 tiles (the global-memory solver)
// Flag the regions holding an active tile.  The flags are zero between
// set-ups (zeroed at allocation, cleared again by k_region_compact), and
// neither kernel runs unless the gate (when given) is set.
__global__ void k_region_flags(const int32_t *__restrict__ n_active,
                               const int32_t *__restrict__ tile_list, RegionGrid g,
                               int32_t *__restrict__ flag, const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  const int na = *n_active;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < na; s += gridDim.x * blockDim.x) {
    const int t = tile_list[s];
    flag[g.region_of_tile(t)] = 1;
  }
}

// Compact the flagged regions (one block): slot of each region (-1 when not
// active), region of each slot, their count, and each slot's six
// neighbouring slots; the flags are cleared behind the read.
__global__ void __launch_bounds__(1024) k_region_compact(RegionGrid g,
                                                         int32_t *__restrict__ flag,
                                                         int32_t *__restrict__ slot,
                                                         int32_t *__restrict__ list,
                                                         int32_t *__restrict__ count,
                                                         int32_t *__restrict__ nbr,
                                                         const int *gate) {
  if (gate != nullptr && *gate == 0) return;
  __shared__ int s_base;
  __shared__ int s_warp[32];
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int r0 = 0; r0 < g.n; r0 += blockDim.x) {
    const int r = r0 + threadIdx.x;
    const int f = r < g.n ? (flag[r] != 0) : 0;
    if (r < g.n && f) flag[r] = 0;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) s_warp[wid] = __popc(m);
    __syncthreads();
    int before = 0;
    for (int w = 0; w < wid; ++w) before += s_warp[w];
    const int k = s_base + before + __popc(m & ((1u << lane) - 1u));
    if (r < g.n) {
      slot[r] = f ? k : -1;
      if (f && k < COARSE_RMAX) list[k] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += s_warp[w];
      s_base += tot;
    }
    __syncthreads();
  }
  const int nr = s_base;
  if (threadIdx.x == 0) *count = nr;
  for (int k = threadIdx.x; k < nr && k < COARSE_RMAX; k += blockDim.x) {
    const int r = list[k];
    const int ri = r / (g.ny * g.nz), rj = (r / g.nz) % g.ny, rk = r % g.nz;
    const int nb[6] = {ri > 0 ? r - g.ny * g.nz : -1, ri < g.nx - 1 ? r + g.ny * g.nz : -1,
                       rj > 0 ? r - g.nz : -1,        rj < g.ny - 1 ? r + g.nz : -1,
                       rk > 0 ? r - 1 : -1,           rk < g.nz - 1 ? r + 1 : -1};
#pragma unroll
    for (int d = 0; d < 6; ++d) nbr[(int64_t)k * 6 + d] = nb[d] >= 0 ? slot[nb[d]] : -1;
  }
}

// Row k of A_c for active region slot k (one block per slot), the slot of
// each of its CT^3 tiles (-1: not active) for the solver's region sums, and
// the region of each of those tile slots.
__global__ void __launch_bounds__(256) k_region_rows(CoarseSetup a, RegionGrid g,
                                                     const int32_t *__restrict__ tile_slot,
                                                     const uint16_t *__restrict__ code,
                                                     int32_t *__restrict__ rtiles,
                                                     int32_t *__restrict__ region_of_slot) {
  const int nr = *a.count;
  const int k = blockIdx.x;
  if (!coarse_active(a, nr) || k >= nr) return;
  const int r = a.ids[k];
  const int ri = r / (g.ny * g.nz), rj = (r / g.nz) % g.ny, rk = r % g.nz;
  const int ct = g.ct, nt3 = ct * ct * ct, span = 8 * ct;
  for (int j = threadIdx.x; j < nt3; j += blockDim.x) {
    const int ti = ri * ct + j / (ct * ct), tj = rj * ct + (j / ct) % ct, tk = rk * ct + j % ct;
    const int sl = ti < g.ntx && tj < g.nty && tk < g.ntz
                       ? tile_slot[((int64_t)ti * g.nty + tj) * g.ntz + tk]
                       : -1;
    rtiles[(int64_t)k * nt3 + j] = sl;
    if (sl >= 0) region_of_slot[sl] = k;
  }
  __syncthreads();
  float v[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int c = threadIdx.x; c < nt3 * 512; c += blockDim.x) {
    const int j = c >> 9, L = c & 511;
    const int sl = rtiles[(int64_t)k * nt3 + j];
    if (sl < 0) continue;
    const uint16_t cd = code[(int64_t)sl * 512 + L];
    if (!(cd & CODE_FLUID)) continue;
    // cell coordinates inside the region
    const int li = (j / (ct * ct)) * 8 + (L >> 6), lj = ((j / ct) % ct) * 8 + ((L >> 3) & 7),
              lk = (j % ct) * 8 + (L & 7);
    int same = 0;
#pragma unroll
    for (int dir = 0; dir < 6; ++dir) {
      if (!(cd & (1 << dir))) continue;
      const bool inside = dir == 0 ? li > 0 : dir == 1 ? li < span - 1 : dir == 2 ? lj > 0
                        : dir == 3 ? lj < span - 1 : dir == 4 ? lk > 0 : lk < span - 1;
      if (inside) ++same; else v[1 + dir] += 1.f;
    }
    v[0] += (float)((int)((cd >> CODE_DIAG_SHIFT) & 7) - same);
  }
  __shared__ float red[8][7];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 7; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    if (lane == 0) red[wid][q] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][threadIdx.x];
    if (threadIdx.x == 0) {
      a.cdiag[k] = t > 0.f ? t : 1.0f;
    } else {
      const int dir = threadIdx.x - 1;
      a.coff[(int64_t)k * 6 + dir] = a.nbr[(int64_t)k * 6 + dir] >= 0 ? -t : 0.f;
    }
  }
}

// ---- row solves (one block per row), written into the B set the last solve
// did not use
__global__ void __launch_bounds__(COARSE_SOLVE_THREADS) k_coarse_solve(CoarseSetup a) {
  extern __shared__ float cs[];  // x, r, p, q: [4][n]
  const int n = *a.count;
  const int row = blockIdx.x;
  if (!coarse_active(a, n) || row >= n) return;
  const CoarseMeta *meta = a.meta;
  const int par = meta->parity;
  const uint16_t *bprev = a.bsets + (int64_t)par * COARSE_RMAX * COARSE_RMAX;
  uint16_t *bh = a.bsets + (int64_t)(par ^ 1) * COARSE_RMAX * COARSE_RMAX;
  // the last B is usable for the warm start when it holds rows of this kind
  const bool have = meta->prev_na > 0 && meta->kind == a.kind;
  const int pr = have ? a.prev_slot[a.ids[row]] : -1;
  float *cx = cs, *cr = cs + n, *cp = cr + n, *cq = cp + n;
  __shared__ float red[COARSE_SOLVE_THREADS / 32][2];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  auto bsum = [&](float a0, float a1, float &o0, float &o1) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, o);
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    }
    if (lane == 0) {
      red[wid][0] = a0;
      red[wid][1] = a1;
    }
    __syncthreads();
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int w = 0; w < COARSE_SOLVE_THREADS / 32; ++w) {
      s0 += red[w][0];
      s1 += red[w][1];
    }
    __syncthreads();
    o0 = s0;
    o1 = s1;
  };
  auto matvec = [&](const float *x, int i) {
    float acc = __ldg(a.cdiag + i) * x[i];
#pragma unroll
    for (int dir = 0; dir < 6; ++dir) {
      const int j = __ldg(a.nbr + (int64_t)i * 6 + dir);
      if (j >= 0 && j < n) acc += __ldg(a.coff + (int64_t)i * 6 + dir) * x[j];
    }
    return acc;
  };
  for (int i = threadIdx.x; i < n; i += blockDim.x) {  // the warm start
    float x0 = 0.f;
    if (pr >= 0) {
      const int pc = a.prev_slot[a.ids[i]];
      if (pc >= 0) x0 = bf16_at(bprev, (int64_t)pr * COARSE_RMAX + pc);
    }
    cx[i] = isfinite(x0) ? x0 : 0.f;
  }
  __syncthreads();
  float rz = 0.f, rn2 = 0.f;
  {
    float a0 = 0.f, a1 = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float b = (i == row ? 1.f : 0.f) - matvec(cx, i);
      cr[i] = b;
      cp[i] = b / __ldg(a.cdiag + i);
      a0 += b * cp[i];
      a1 += b * b;
    }
    bsum(a0, a1, rz, rn2);
  }
  bool ok = rn2 <= kCoarseTol2;
  for (int it = 0; it < 1000 && !ok; ++it) {
    float pq, dummy;
    {
      float a0 = 0.f;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = matvec(cp, i);
        cq[i] = v;
        a0 += cp[i] * v;
      }
      bsum(a0, 0.f, pq, dummy);
    }
    if (!(pq > 0.f)) break;
    const float al = rz / pq;
    float a0 = 0.f, a1 = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      cx[i] += al * cp[i];
      const float rn = cr[i] - al * cq[i];
      cr[i] = rn;
      a0 += rn * rn;
      a1 += rn * rn / __ldg(a.cdiag + i);
    }
    float rz2;
    bsum(a0, a1, rn2, rz2);
    if (rn2 <= kCoarseTol2) {
      ok = true;
      break;
    }
    const float be = rz2 / rz;
    rz = rz2;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      cp[i] = cr[i] / __ldg(a.cdiag + i) + be * cp[i];
    __syncthreads();
  }
  bool finite = true;
  uint16_t *out = bh + (int64_t)row * COARSE_RMAX;
  const int n8 = (n + 7) & ~7;
  for (int i = threadIdx.x; i < n8; i += blockDim.x) {
    const float x = i < n ? cx[i] : 0.f;
    finite &= isfinite(x);
    out[i] = __bfloat16_as_ushort(__float2bfloat16_rn(x));
  }
  if ((threadIdx.x == 0 && !ok) || !finite) atomicExch(&a.st->coarse_off, 1);
}

// After the row solves: the id-to-row map and the row ids describe the new
// B, and the parity names its set.  First the last B's ids lose their rows,
// then the new ones get theirs (two launches, so that no block clears an
// entry another has already set).
__global__ void k_coarse_commit_clear(CoarseSetup a) {
  const int n = *a.count;
  if (!coarse_active(a, n)) return;
  const CoarseMeta *meta = a.meta;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < meta->prev_na;
       s += gridDim.x * blockDim.x)
    a.prev_slot[a.prev_list[s]] = -1;
}
__global__ void k_coarse_commit_set(CoarseSetup a) {
  const int n = *a.count;
  if (!coarse_active(a, n)) return;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const int id = a.ids[s];
    a.prev_slot[id] = s;
    a.prev_list[s] = id;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.meta->prev_na = n;
    a.meta->kind = a.kind;
    a.meta->parity ^= 1;
  }
}

static CoarseSetup coarse_args(Ctx *c, const int32_t *count, const int32_t *ids,
                               const int32_t *nbr, PcgState *st, int limit, const int *gate,
                               int kind) {
  unsigned char *b = c->coarse_buf;
  CoarseSetup a;
  a.count = count;
  a.ids = ids;
  a.nbr = nbr;
  a.cdiag = reinterpret_cast<float *>(b + COARSE_DIAG_OFF);
  a.coff = reinterpret_cast<float *>(b + COARSE_OFF_OFF);
  a.bsets = reinterpret_cast<uint16_t *>(b);
  a.prev_slot = c->coarse_prev_slot;
  a.prev_list = reinterpret_cast<int32_t *>(b + COARSE_LIST_OFF);
  a.meta = reinterpret_cast<CoarseMeta *>(b + COARSE_META_OFF);
  a.st = st;
  a.limit = limit;
  a.gate = gate;
  a.kind = kind;
  return a;
}

static int coarse_solve_and_commit(Ctx *c, const CoarseSetup &a) {
  const size_t vec = (size_t)4 * COARSE_RMAX * sizeof(float);
  k_coarse_solve<<<COARSE_RMAX, COARSE_SOLVE_THREADS, vec, c->stream>>>(a);
  k_coarse_commit_clear<<<(COARSE_RMAX + 255) / 256, 256, 0, c->stream>>>(a);
  k_coarse_commit_set<<<(COARSE_RMAX + 255) / 256, 256, 0, c->stream>>>(a);
  c->launches += 3;
  return check_launch(c, "coarse correction set-up");
}

int coarse_setup_tiles(Ctx *c, const int32_t *n_active, const int32_t *tile_list,
                       const int32_t *tile_nbr, const uint16_t *code, PcgState *st, int limit) {
  const CoarseSetup a = coarse_args(c, n_active, tile_list, tile_nbr, st, limit, nullptr,
                                    COARSE_KIND_TILES);
  k_coarse_tile_rows<<<COARSE_RMAX, 256, 0, c->stream>>>(a, code);
  c->launches++;
  return coarse_solve_and_commit(c, a);
}

RegionBufs region_bufs(Ctx *c) {
  const RegionGrid &g = c->rg;
  RegionBufs b;
  b.flag = c->rg_buf;
  b.slot = b.flag + g.n;
  b.list = b.slot + g.n;
  b.count = b.list + COARSE_RMAX;
  b.nbr = b.count + 4;
  b.tiles = b.nbr + (int64_t)COARSE_RMAX * 6;
  b.of_slot = b.tiles + (int64_t)COARSE_RMAX * g.ct * g.ct * g.ct;
  return b;
}

int coarse_setup_regions(Ctx *c, PcgState *st, const int *gate) {
  const RegionGrid g = c->rg;
  const RegionBufs b = region_bufs(c);
  int32_t *flag = b.flag, *slot = b.slot, *list = b.list, *count = b.count, *nbr = b.nbr,
          *rtiles = b.tiles;
  k_region_flags<<<c->num_sms * 4, 256, 0, c->stream>>>(c->n_active, c->tile_list, g, flag,
                                                        gate);
  k_region_compact<<<1, 1024, 0, c->stream>>>(g, flag, slot, list, count, nbr, gate);
  const CoarseSetup a =
      coarse_args(c, count, list, nbr, st, COARSE_RMAX, gate, COARSE_KIND_REGIONS);
  k_region_rows<<<COARSE_RMAX, 256, 0, c->stream>>>(a, g, c->tile_slot, c->code, rtiles,
                                                    b.of_slot);
  c->launches += 3;
  return coarse_solve_and_commit(c, a);
}

}  // namespace gf
