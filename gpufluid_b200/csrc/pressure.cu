// Pressure projection on a compact array of active 8x8x8 tiles.
//
// Set-up (once per solve):
//   k_tile_flags    tile active iff it holds a fluid cell (k_mark_active_blocks,
//                   solver3d.py:953-972)
//   k_tile_compact  slot numbering of active tiles along a Morton curve (the reference's
//                   array_scan + k_compact_active_blocks, :1056-1082)
//   k_tile_setup    neighbour-tile table, per-cell 16-bit stencil code
//                   (fluid-neighbour mask + #non-solid neighbours), compact rhs
// Solvers:
//   k_jacobi        one sweep of k3_jacobi_pressure (:878-938)
//   k_gsrb          one colour of k3_gauss_seidel_rb (:1204-1267)
//   k_pcg<Acc,REF,SGS>  the whole preconditioned CG of _pressure_pcg
//                   (:2917-3043; the reference's Jacobi preconditioner, or with
//                   SGS the tile-local symmetric Gauss-Seidel one of the
//                   shared-memory solver) in ONE persistent cooperative kernel: two
//                   grid barriers per iteration, dot products reduced
//                   warp -> block -> fixed-order last-block sum (deterministic),
//                   convergence decided on the device.  REF=true adds FP64
//                   residual replacement: x accumulates in FP64 and, whenever
//                   the FP32 recursive residual has dropped by a fixed factor,
//                   r is recomputed as b - A x in FP64 (the only FP64 work
//                   besides the FP64 dot-product accumulation).
//   k_scatter_p     compact solution -> dense p (non-fluid cells stay 0)
//
// Every spin-wait (grid barrier) is bounded; on timeout the kernel records
// GF_TIMEOUT in the solve state and all blocks return.
#include <algorithm>
#include <utility>
#include <vector>

#include "gf_internal.cuh"

namespace gf {

constexpr int PCG_THREADS = 512;
constexpr size_t BAR_BYTES = 8 * 16 * 8;  // barrier scratch: 8 lines x 16 u64
constexpr long long SPIN_LIMIT = 1LL << 24;  // ~1-2 s with 64 ns sleeps

// ------------------------------------------------------------- set-up
__global__ void k_tile_flags(const uint8_t *__restrict__ label, int nx, int ny, int nz,
                             int nty, int ntz, int ntiles, int32_t *__restrict__ flag) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ntiles) return;
  int ti = warp / (nty * ntz), tj = (warp / ntz) % nty, tk = warp % ntz;
  int any = 0;
  for (int row = lane; row < 64; row += 32) {
    int gi = ti * 8 + (row >> 3), gj = tj * 8 + (row & 7);
    if (gi >= nx || gj >= ny) continue;
    const uint8_t *base = label + ((int64_t)gi * ny + gj) * nz;
    for (int lk = 0; lk < 8; ++lk) {
      int gk = tk * 8 + lk;
      if (gk < nz && base[gk] == 1) any = 1;
    }
  }
  any = __any_sync(0xffffffffu, any);
  if (lane == 0) flag[warp] = any;
}

// Slots follow `order` (a permutation of the tile ids; identity when NULL):
// the single-grid solvers number active tiles along a Morton curve, so that
// contiguous slot runs -- the units the PCG blocks own -- are compact 3-D
// clusters with few faces on another block's tiles.
__global__ void k_tile_compact(const int32_t *__restrict__ flag, int ntiles,
                               const int32_t *__restrict__ order, int32_t *__restrict__ slot,
                               int32_t *__restrict__ list, int32_t *__restrict__ n_active) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int off = 0; off < ntiles; off += blockDim.x) {
    const int i = off + threadIdx.x;
    const int t = i < ntiles ? (order ? order[i] : i) : ntiles;
    int f = i < ntiles ? flag[t] : 0;
    int incl = f;
    for (int o = 1; o < 32; o <<= 1) {
      int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (unsigned)o) incl += v;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int s = lane < nw ? warp_sums[lane] : 0, si = s;
      for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= (unsigned)o) si += v;
      }
      if (lane < nw) warp_sums[lane] = si - s;
    }
    __syncthreads();
    int pre = carry + warp_sums[wid] + incl - f;
    if (i < ntiles) {
      slot[t] = f ? pre : -1;
      if (f) list[pre] = t;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = pre + f;
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_active = carry;
}

struct SetupArgs {
  const uint8_t *label;
  const float *div;
  const int32_t *n_active, *tile_list, *tile_slot;
  int32_t *tile_nbr;
  uint16_t *code;
  float *bdiv, *x, *r, *z, *d0, *d1, *Ad;
  double *x64;
  int64_t *n_fluid;
  int32_t *tile_cost;  // per slot: fluid cells + 192 (work estimate of the PCG)
  int nx, ny, nz, ntx, nty, ntz;
};

__global__ void __launch_bounds__(512) k_tile_setup(SetupArgs a) {
  const int na = *a.n_active;
  const int l = threadIdx.x, li = l >> 6, lj = (l >> 3) & 7, lk = l & 7;
  for (int s = blockIdx.x; s < na; s += gridDim.x) {
    const int t = a.tile_list[s];
    const int ti = t / (a.nty * a.ntz), tj = (t / a.ntz) % a.nty, tk = t % a.ntz;
    if (l < 6) {
      int ni = ti + (l == 0 ? -1 : l == 1 ? 1 : 0), nj = tj + (l == 2 ? -1 : l == 3 ? 1 : 0),
          nk = tk + (l == 4 ? -1 : l == 5 ? 1 : 0);
      int ns = -1;
      if (ni >= 0 && ni < a.ntx && nj >= 0 && nj < a.nty && nk >= 0 && nk < a.ntz)
        ns = a.tile_slot[(ni * a.nty + nj) * a.ntz + nk];
      a.tile_nbr[s * 6 + l] = ns;
    }
    const int gi = ti * 8 + li, gj = tj * 8 + lj, gk = tk * 8 + lk;
    const int64_t q = (int64_t)s * TILE_CELLS + l;
    uint16_t code = 0;
    float bd = 0.f;
    if (gi < a.nx && gj < a.ny && gk < a.nz) {
      const int ny = a.ny, nz = a.nz;
      const int64_t c = ((int64_t)gi * ny + gj) * nz + gk;
      if (a.label[c] == 1) {
        int diag = 0, mask = 0, m;
        // neighbour order -x, +x, -y, +y, -z, +z as in the reference stencil
        if (gi > 0) { m = a.label[c - (int64_t)ny * nz]; if (m != 2) { ++diag; if (m == 1) mask |= 1; } }
        if (gi < a.nx - 1) { m = a.label[c + (int64_t)ny * nz]; if (m != 2) { ++diag; if (m == 1) mask |= 2; } }
        if (gj > 0) { m = a.label[c - nz]; if (m != 2) { ++diag; if (m == 1) mask |= 4; } }
        if (gj < ny - 1) { m = a.label[c + nz]; if (m != 2) { ++diag; if (m == 1) mask |= 8; } }
        if (gk > 0) { m = a.label[c - 1]; if (m != 2) { ++diag; if (m == 1) mask |= 16; } }
        if (gk < nz - 1) { m = a.label[c + 1]; if (m != 2) { ++diag; if (m == 1) mask |= 32; } }
        code = (uint16_t)(CODE_FLUID | (diag << CODE_DIAG_SHIFT) | mask);
        bd = a.div[c];
      }
    }
    {
      const int nf = __syncthreads_count(code != 0);
      if (l == 0) a.tile_cost[s] = nf + 192;
      if (l == 0 && nf) atomicAdd(reinterpret_cast<unsigned long long *>(a.n_fluid),
                                 (unsigned long long)nf);
    }
    a.code[q] = code;
    a.bdiv[q] = bd;
    a.x[q] = 0.f;
    a.r[q] = 0.f;
    a.z[q] = 0.f;
    a.d0[q] = 0.f;
    a.d1[q] = 0.f;
    a.Ad[q] = 0.f;
    if (a.x64) a.x64[q] = 0.0;
  }
}

// ---- set-up over a batch: tiles are numbered scene after scene, so the
// compaction keeps every scene's active tiles in one contiguous slot range.
__global__ void kb_tile_flags(const uint8_t *__restrict__ label, SegIndex sx, int64_t ntiles,
                              int32_t *__restrict__ flag) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ntiles) return;
  const SegRow r = sx.row[seg_find(sx.tile0, sx.n, warp)];
  const int t = (int)(warp - r.tile0);
  const int ti = t / (r.nty * r.ntz), tj = (t / r.ntz) % r.nty, tk = t % r.ntz;
  const uint8_t *lab = label + r.cell0;
  int any = 0;
  for (int row = lane; row < 64; row += 32) {
    int gi = ti * 8 + (row >> 3), gj = tj * 8 + (row & 7);
    if (gi >= r.nx || gj >= r.ny) continue;
    const uint8_t *base = lab + ((int64_t)gi * r.ny + gj) * r.nz;
    for (int lk = 0; lk < 8; ++lk) {
      int gk = tk * 8 + lk;
      if (gk < r.nz && base[gk] == 1) any = 1;
    }
  }
  any = __any_sync(0xffffffffu, any);
  if (lane == 0) flag[warp] = any;
}

// First active slot of every scene (slot0[nseg] = number of active tiles).
__global__ void kb_slot_ranges(const int32_t *__restrict__ tile_list,
                               const int32_t *__restrict__ n_active, SegIndex sx,
                               int32_t *__restrict__ slot0) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s > sx.n) return;
  const int na = *n_active;
  if (s == sx.n) {
    slot0[s] = na;
    return;
  }
  const int64_t t0 = sx.tile0[s];
  int lo = 0, hi = na;  // first slot whose tile >= t0
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tile_list[mid] < t0) lo = mid + 1; else hi = mid;
  }
  slot0[s] = lo;
}

struct BatchSetupArgs {
  SetupArgs a;  // label/div are the concatenated arrays; grid fields unused
  SegIndex sx;
};

__global__ void __launch_bounds__(512) kb_tile_setup(BatchSetupArgs ba) {
  const SetupArgs &a = ba.a;
  const int na = *a.n_active;
  const int l = threadIdx.x, li = l >> 6, lj = (l >> 3) & 7, lk = l & 7;
  for (int s = blockIdx.x; s < na; s += gridDim.x) {
    const int tg = a.tile_list[s];
    const SegRow r = ba.sx.row[seg_find(ba.sx.tile0, ba.sx.n, tg)];
    const int t = (int)(tg - r.tile0);
    const int ti = t / (r.nty * r.ntz), tj = (t / r.ntz) % r.nty, tk = t % r.ntz;
    if (l < 6) {
      int ni = ti + (l == 0 ? -1 : l == 1 ? 1 : 0), nj = tj + (l == 2 ? -1 : l == 3 ? 1 : 0),
          nk = tk + (l == 4 ? -1 : l == 5 ? 1 : 0);
      int ns = -1;
      if (ni >= 0 && ni < r.ntx && nj >= 0 && nj < r.nty && nk >= 0 && nk < r.ntz)
        ns = a.tile_slot[r.tile0 + (ni * r.nty + nj) * r.ntz + nk];
      a.tile_nbr[s * 6 + l] = ns;
    }
    const int gi = ti * 8 + li, gj = tj * 8 + lj, gk = tk * 8 + lk;
    const int64_t q = (int64_t)s * TILE_CELLS + l;
    uint16_t code = 0;
    float bd = 0.f;
    if (gi < r.nx && gj < r.ny && gk < r.nz) {
      const int nx = r.nx, ny = r.ny, nz = r.nz;
      const uint8_t *lab = a.label + r.cell0;
      const int64_t c = ((int64_t)gi * ny + gj) * nz + gk;
      if (lab[c] == 1) {
        int diag = 0, mask = 0, m;
        if (gi > 0) { m = lab[c - (int64_t)ny * nz]; if (m != 2) { ++diag; if (m == 1) mask |= 1; } }
        if (gi < nx - 1) { m = lab[c + (int64_t)ny * nz]; if (m != 2) { ++diag; if (m == 1) mask |= 2; } }
        if (gj > 0) { m = lab[c - nz]; if (m != 2) { ++diag; if (m == 1) mask |= 4; } }
        if (gj < ny - 1) { m = lab[c + nz]; if (m != 2) { ++diag; if (m == 1) mask |= 8; } }
        if (gk > 0) { m = lab[c - 1]; if (m != 2) { ++diag; if (m == 1) mask |= 16; } }
        if (gk < nz - 1) { m = lab[c + 1]; if (m != 2) { ++diag; if (m == 1) mask |= 32; } }
        code = (uint16_t)(CODE_FLUID | (diag << CODE_DIAG_SHIFT) | mask);
        bd = a.div[r.cell0 + c];
      }
    }
    {
      const int nf = __syncthreads_count(code != 0);
      if (l == 0) a.tile_cost[s] = nf + 192;
      if (l == 0 && nf) atomicAdd(reinterpret_cast<unsigned long long *>(a.n_fluid),
                                 (unsigned long long)nf);
    }
    a.code[q] = code;
    a.bdiv[q] = bd;
    a.x[q] = 0.f;
    a.r[q] = 0.f;
    a.z[q] = 0.f;
    a.d0[q] = 0.f;
    a.d1[q] = 0.f;
    a.Ad[q] = 0.f;
    if (a.x64) a.x64[q] = 0.0;
  }
}

// Compact index of neighbour `dir` (0 -x, 1 +x, 2 -y, 3 +y, 4 -z, 5 +z) of q.
// Only called for fluid neighbours, whose tile is active by construction.
__device__ __forceinline__ int64_t nb_index(int64_t q, int dir, const int32_t *__restrict__ nbr) {
  const int s = (int)(q >> 9), l = (int)(q & 511);
  const int li = l >> 6, lj = (l >> 3) & 7, lk = l & 7;
  switch (dir) {
    case 0: return li > 0 ? q - 64 : (int64_t)__ldg(nbr + s * 6 + 0) * 512 + (448 | (l & 63));
    case 1: return li < 7 ? q + 64 : (int64_t)__ldg(nbr + s * 6 + 1) * 512 + (l & 63);
    case 2: return lj > 0 ? q - 8 : (int64_t)__ldg(nbr + s * 6 + 2) * 512 + ((l & 0x1C7) | 56);
    case 3: return lj < 7 ? q + 8 : (int64_t)__ldg(nbr + s * 6 + 3) * 512 + (l & 0x1C7);
    case 4: return lk > 0 ? q - 1 : (int64_t)__ldg(nbr + s * 6 + 4) * 512 + (l | 7);
    default: return lk < 7 ? q + 1 : (int64_t)__ldg(nbr + s * 6 + 5) * 512 + (l & ~7);
  }
}

// ------------------------------------------------------------- Jacobi / GS
struct SweepArgs {
  const int32_t *n_active, *nbr;
  const uint16_t *code;
  const float *bdiv;
};

__global__ void k_jacobi(SweepArgs a, const float *__restrict__ xin, float *__restrict__ xout) {
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint16_t code = a.code[q];
    if (!(code & CODE_FLUID)) continue;  // stays 0
    float s = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; ++d)
      if (code & (1 << d)) {
        const int64_t nq = nb_index(q, d, a.nbr);
        if (GF_IN(nq, total)) s = s + xin[nq];
      }
    const float diag = (float)((code >> CODE_DIAG_SHIFT) & 7);
    xout[q] = diag < 0.5f ? 0.0f : (s - a.bdiv[q]) / diag;
  }
}

__global__ void k_gsrb(SweepArgs a, float *__restrict__ x, int color) {
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(q & 511);
    if ((((l >> 6) + ((l >> 3) & 7) + (l & 7)) & 1) != color) continue;  // global parity
    const uint16_t code = a.code[q];
    if (!(code & CODE_FLUID)) continue;
    float s = 0.0f;
#pragma unroll
    for (int d = 0; d < 6; ++d)
      if (code & (1 << d)) {
        const int64_t nq = nb_index(q, d, a.nbr);
        if (GF_IN(nq, total)) s = s + x[nq];
      }
    const float diag = (float)((code >> CODE_DIAG_SHIFT) & 7);
    x[q] = diag < 0.5f ? 0.0f : (s - a.bdiv[q]) / diag;
  }
}

// ------------------------------------------------------------------ PCG
struct PcgArgs {
  const int32_t *n_active, *nbr;
  const uint16_t *code;
  const float *bdiv;
  float *x, *r, *z, *d0, *d1, *Ad;
  double *x64;
  double *partials;
  PcgState *st;
  int max_iter, check_every;
  double tol2;     // tol^2
  double replace2; // residual-replacement factor^2 (refined)
  float sign;      // b = sign * div
  int only_if_fallback;  // run only when the shared-memory solver deferred
  int sgs;         // tile-local symmetric Gauss-Seidel sweeps (SGS instantiation)
  // warm start (refined only): x64 starts at the dense pressure p0 of the
  // previous solve; the tile list and grid sizes map a slot to its cell of p0
  int warm;
  const float *p0;
  const int32_t *tile_list;
  int ny, nz, nty, ntz;
  // cube-region coarse correction (SGS instantiation; coarse.cu set up its
  // rows): active regions, the tile slots of each region [RMAX][ct^3], the
  // region of each tile slot, the tiles' residual sums, the corrections e
  int coarse;
  const int32_t *rg_count, *rg_tiles, *rg_of_slot;
  int rg_nt3;
  float *rg_gt, *rg_e;
  const unsigned char *cbuf;
};

// ---- tile-local symmetric Gauss-Seidel preconditioner of the global-memory
// PCG: z = M^-1 r with M^-1 = `sgs` red-black symmetric Gauss-Seidel sweeps
// on each 8^3 tile from z = r / D, the tile's neighbours held at zero (the
// diagonal block of A per tile: symmetric positive definite, so CG applies).
// The same preconditioner as the shared-memory solver's.  A block takes
// SGS_TB tiles per round: each thread owns local cell `tid` of every tile of
// the round for the update, then the half-sweeps run in shared memory on
// 10^3 padded boxes whose one-cell ring stays zero.
constexpr int SGS_TB = 4;
struct SgsSmem {
  float zb[SGS_TB * 1000];
  float r[SGS_TB * 512];
  uint16_t code[SGS_TB * 512];
};

__device__ __forceinline__ int tile_pad(int l) {
  return ((l >> 6) + 1) * 100 + (((l >> 3) & 7) + 1) * 10 + ((l & 7) + 1);
}
__device__ __forceinline__ float sgs_factor(unsigned code) {  // 1 / max(D, 1) on fluid, else 0
  return (code & CODE_FLUID) ? 1.0f / fmaxf((float)((code >> CODE_DIAG_SHIFT) & 7), 1.0f) : 0.0f;
}
// z = (r + the in-tile fluid neighbours' z) / D on colour c of the round's
// tiles (thread t: cell sgs_color_cell(t & 255, c) in tiles t >> 8, +2).
__device__ __forceinline__ void sgs_half(SgsSmem &S, int c) {
  const int lc = sgs_color_cell(threadIdx.x & 255, c), pc = tile_pad(lc);
  for (int m = threadIdx.x >> 8; m < SGS_TB; m += PCG_THREADS / 256) {
    float *zp = S.zb + m * 1000 + pc;
    float acc = S.r[m * 512 + lc];
    acc = acc + zp[-100];
    acc = acc + zp[100];
    acc = acc + zp[-10];
    acc = acc + zp[10];
    acc = acc + zp[-1];
    acc = acc + zp[1];
    *zp = acc * sgs_factor(S.code[m * 512 + lc]);
  }
}
// After the round's r and code are in S (and z = r / D in the boxes): the
// sweeps; the caller then reads z of its cells from S.zb.
__device__ __forceinline__ void sgs_sweeps(SgsSmem &S, int sweeps) {
  __syncthreads();
  for (int sw = 0; sw < sweeps; ++sw) {
    sgs_half(S, 1);
    __syncthreads();
    sgs_half(S, 0);
    __syncthreads();
  }
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
  // deterministic: fixed shuffle tree, then warp 0 sums the per-warp values
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  T t = 0;
  if (wid == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : (T)0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  __syncthreads();
  return t;  // valid in thread 0
}

__device__ __forceinline__ unsigned ld_volatile(const unsigned *p) {
  return *reinterpret_cast<const volatile unsigned *>(p);
}
__device__ __forceinline__ int ld_volatile_i(const int *p) {
  return *reinterpret_cast<const volatile int *>(p);
}
__device__ __forceinline__ double ld_volatile_d(const double *p) {
  return *reinterpret_cast<const volatile double *>(p);
}

// Grid-wide reduction of NV values + barrier.  Every block writes its block
// sums to partials; the last block to arrive sums all partials in a fixed
// order, runs `fin` (thread 0) on the totals, then releases the others.
// Returns false when a wait timed out (the caller must return).
template <typename T, int NV, typename Fin>
__device__ bool grid_reduce(const PcgArgs &a, T (&v)[NV], Fin fin) {
  __shared__ T sh[32];
  __shared__ int s_last, s_ok;
  T tot[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) tot[k] = block_sum<T>(v[k], sh);
  const unsigned nb = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) a.partials[k * MAX_PCG_BLOCKS + blockIdx.x] = (double)tot[k];
  }
  __syncthreads();
  unsigned gen = 0;
  if (threadIdx.x == 0) {
    gen = ld_volatile(&a.st->bar_gen);
    __threadfence();
    unsigned arrived = atomicAdd(&a.st->bar_count, 1u);
    s_last = arrived == nb - 1;
    s_ok = 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    double all[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      T acc = 0;
      for (unsigned j = threadIdx.x; j < nb; j += blockDim.x)
        acc += (T)__ldcg(a.partials + k * MAX_PCG_BLOCKS + j);
      all[k] = (double)block_sum<T>(acc, sh);
    }
    if (threadIdx.x == 0) {
      fin(all);
      __threadfence();
      atomicExch(&a.st->bar_count, 0u);
      __threadfence();
      atomicAdd(&a.st->bar_gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    long long spins = 0;
    while (ld_volatile(&a.st->bar_gen) == gen) {
      if (++spins > SPIN_LIMIT) {
        atomicExch(&a.st->error, 1);
        s_ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
  if (ld_volatile_i(&a.st->error)) return false;
  return s_ok;
}

__device__ bool grid_barrier(const PcgArgs &a) {
  double v[1] = {0.0};
  return grid_reduce<double, 1>(a, v, [](double *) {});
}

template <typename Acc, bool REF, bool SGS>
__global__ void __launch_bounds__(PCG_THREADS, 2) k_pcg(PcgArgs a) {
  if (a.only_if_fallback && !ld_volatile_i(&a.st->fallback)) return;
  __shared__ alignas(16) unsigned char sgs_raw[SGS ? sizeof(SgsSmem) : 16];
  SgsSmem &S = *reinterpret_cast<SgsSmem *>(sgs_raw);  // boxes of the SGS instantiation
  const int na = *a.n_active;
  // cube-region coarse correction (tile SGS only): u = z + P e with
  // e = B P^T r, B's bf16 rows from the set-up; off when a row solve failed
  // or the set-up did not run (too many regions)
  __shared__ float s_g[SGS ? COARSE_RMAX : 1];   // every region's residual sum
  __shared__ float s_tp[SGS ? SGS_TB * 16 : 1];  // warp partials of the round's tile sums
  const int nreg = SGS && a.coarse ? *a.rg_count : 0;
  const bool coarse = SGS && a.coarse && nreg > 0 && nreg <= COARSE_RMAX &&
                      ld_volatile_i(&a.st->coarse_off) == 0;
  const uint16_t *Bh = nullptr;
  if (coarse)
    Bh = reinterpret_cast<const uint16_t *>(a.cbuf) +
         (int64_t)reinterpret_cast<const CoarseMeta *>(a.cbuf + COARSE_META_OFF)->parity *
             COARSE_RMAX * COARSE_RMAX;
  // tile sums of r over a round's SGS_TB tiles (thread t holds cell t of each)
  auto tile_sums = [&](int base, const float (&v)[SGS_TB]) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < SGS_TB; ++m) {
      float x = v[m];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) s_tp[m * 16 + wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < SGS_TB && base + (int)threadIdx.x < na) {
      float s = 0.f;
#pragma unroll
      for (int w = 0; w < 16; ++w) s += s_tp[threadIdx.x * 16 + w];
      a.rg_gt[base + threadIdx.x] = s;
    }
  };
  // the coarse correction of e = B P^T r after a grid barrier that follows
  // the tile sums: every block sums all regions' g into shared memory (the
  // region's tiles in index order), its warps form e for a share of the
  // regions, and g . e = r . P e rides on one grid reduction whose `fin`
  // gets the total
  auto coarse_step = [&](auto fin) -> bool {
    for (int k = threadIdx.x; k < nreg; k += blockDim.x) {
      float g = 0.f;
      for (int j = 0; j < a.rg_nt3; ++j) {
        const int sl = a.rg_tiles[(int64_t)k * a.rg_nt3 + j];
        if (sl >= 0) g += __ldcg(a.rg_gt + sl);
      }
      s_g[k] = g;
    }
    for (int k = nreg + threadIdx.x; k < ((nreg + 7) & ~7); k += blockDim.x) s_g[k] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double ge = 0.0;
    for (int k = blockIdx.x * nw + wid; k < nreg; k += gridDim.x * nw) {
      const uint4 *row = reinterpret_cast<const uint4 *>(Bh + (int64_t)k * COARSE_RMAX);
      float v = 0.f;
      for (int ch = lane; ch < ((nreg + 7) >> 3); ch += 32) {
        const uint4 q = __ldg(row + ch);
        const float *gp = s_g + ch * 8;
        v += __uint_as_float(q.x << 16) * gp[0] + __uint_as_float(q.x & 0xffff0000u) * gp[1];
        v += __uint_as_float(q.y << 16) * gp[2] + __uint_as_float(q.y & 0xffff0000u) * gp[3];
        v += __uint_as_float(q.z << 16) * gp[4] + __uint_as_float(q.z & 0xffff0000u) * gp[5];
        v += __uint_as_float(q.w << 16) * gp[6] + __uint_as_float(q.w & 0xffff0000u) * gp[7];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) {
        a.rg_e[k] = v;
        ge += (double)s_g[k] * (double)v;
      }
    }
    double w[1] = {ge};
    return grid_reduce<double, 1>(a, w, fin);
  };
  // u = z + e of the cell's region
  auto ecell = [&](int64_t q) -> float {
    return coarse ? __ldcg(a.rg_e + a.rg_of_slot[q >> 9]) : 0.0f;
  };
  if (SGS) {  // the boxes' rings stay zero for the whole solve
    for (int q = threadIdx.x; q < SGS_TB * 1000; q += blockDim.x) S.zb[q] = 0.f;
  }
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t q0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  PcgState *st = a.st;
  constexpr int KQ = 4;
  float *__restrict__ X = a.x;
  float *__restrict__ R = a.r;
  float *__restrict__ Z = a.z;
  float *__restrict__ AD = a.Ad;
  const uint16_t *__restrict__ CODE = a.code;

  // ---- init: x = 0, r = b, z = M^-1 r, d = 0 (so the first d = z).  With
  // the warm start (refined only) x64 = p0 at each fluid cell and r = b - A p0
  // in FP64 from the dense p0 (complete and read-only during the solve); the
  // stop test stays relative to ||b||, so the accuracy target is unchanged.
  const bool warm = REF && a.warm && a.p0 != nullptr;
  double wb2 = 0.0, wr2 = 0.0;  // this thread's sums of b^2 and (b - A p0)^2
  auto warm_residual = [&](int64_t q, uint16_t code, float b) -> float {
    const int t = a.tile_list[q >> 9];
    const int l = (int)(q & 511);
    const int ti = t / (a.nty * a.ntz), tj = (t / a.ntz) % a.nty, tk = t % a.ntz;
    const int64_t sI = (int64_t)a.ny * a.nz;
    const int64_t g = (int64_t)(ti * 8 + (l >> 6)) * sI + (tj * 8 + ((l >> 3) & 7)) * a.nz +
                      (tk * 8 + (l & 7));
    const double x0 = (double)a.p0[g];
    const int64_t off[6] = {-sI, sI, -(int64_t)a.nz, (int64_t)a.nz, -1, 1};
    double sum = 0.0;
#pragma unroll
    for (int dir = 0; dir < 6; ++dir)
      if (code & (1 << dir)) sum += (double)a.p0[g + off[dir]];
    const double res = (double)b - ((double)((code >> CODE_DIAG_SHIFT) & 7) * x0 - sum);
    a.x64[q] = x0;
    wb2 += (double)b * (double)b;
    wr2 += res * res;
    return (float)res;
  };
  {
    Acc v[2] = {0, 0};
    if (SGS) {
      const int tid = threadIdx.x;
      for (int base = blockIdx.x * SGS_TB; base < na; base += gridDim.x * SGS_TB) {
        float bb[SGS_TB];
#pragma unroll
        for (int m = 0; m < SGS_TB; ++m) {
          const int64_t q = (int64_t)(base + m) * 512 + tid;
          const uint16_t code = base + m < na ? CODE[q] : (uint16_t)0;
          bb[m] = (code & CODE_FLUID) ? a.sign * a.bdiv[q] : 0.0f;
          if (warm && (code & CODE_FLUID)) bb[m] = warm_residual(q, code, bb[m]);
          if (code & CODE_FLUID) a.r[q] = bb[m];
          S.r[m * 512 + tid] = bb[m];
          S.code[m * 512 + tid] = code;
          S.zb[m * 1000 + tile_pad(tid)] = bb[m] * sgs_factor(code);
        }
        sgs_sweeps(S, a.sgs);
#pragma unroll
        for (int m = 0; m < SGS_TB; ++m) {
          if (!(S.code[m * 512 + tid] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m) * 512 + tid;
          const float z = S.zb[m * 1000 + tile_pad(tid)];
          a.z[q] = z;
          v[0] += (Acc)(bb[m] * z);
          v[1] += (Acc)(bb[m] * bb[m]);
        }
        if (coarse) tile_sums(base, bb);
        __syncthreads();
      }
    } else {
      for (int64_t q = q0; q < total; q += stride) {
        const uint16_t code = a.code[q];
        if (!(code & CODE_FLUID)) continue;
        float b = a.sign * a.bdiv[q];
        if (warm) b = warm_residual(q, code, b);
        const float diag = fmaxf((float)((code >> CODE_DIAG_SHIFT) & 7), 1.0f);
        const float z = b / diag;
        a.r[q] = b;
        a.z[q] = z;
        v[0] += (Acc)(b * z);
        v[1] += (Acc)(b * b);
      }
    }
    if (warm) {
      double w[2] = {wb2, wr2};
      if (!grid_reduce<double, 2>(a, w, [&](double *t) {
            st->b2 = t[0];
            st->r_true2 = t[1];
          }))
        return;
    }
    if (!grid_reduce<Acc, 2>(a, v, [&](double *t) {
          st->rz = t[0];
          st->rz_part = t[0];
          st->r0 = t[1];
          st->rr = t[1];
          st->r_upd2 = t[1];
          st->beta = 0.0;
          st->alpha = 0.0;
          st->iters = 0;
          st->n_replace = 0;
          st->status = GF_OK;
          if (warm) {
            const double b2 = ld_volatile_d(&st->b2), rt2 = ld_volatile_d(&st->r_true2);
            st->done = b2 < 1e-30 || rt2 <= a.tol2 * b2 ? 1 : 0;
          } else {
            st->b2 = t[1];
            st->r_true2 = t[1];
            st->done = t[1] < 1e-30 ? 1 : 0;  // the reference's early exit (:2982-2986)
          }
        }))
      return;
    if (coarse && !coarse_step([&](double *t) { st->rz = st->rz_part + t[0]; })) return;
  }

  for (int it = 0; it < a.max_iter; ++it) {
    if (ld_volatile_i(&st->done)) break;
    const float beta = (float)ld_volatile_d(&st->beta);
    const float *__restrict__ dold = (it & 1) ? a.d1 : a.d0;
    float *__restrict__ dnew = (it & 1) ? a.d0 : a.d1;
    // ---- phase A: d = z + beta d ; Ad = A d ; p.Ap
    // (KQ cells per thread per step: every load of the step is issued before
    // its stores, so the step's loads are in flight together)
    {
      Acc v[1] = {0};
      for (int64_t qb = q0; qb < total; qb += KQ * stride) {
        uint16_t cd[KQ];
        float dn[KQ], sn[KQ];
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          const int64_t q = qb + m * stride;
          cd[m] = q < total ? CODE[q] : (uint16_t)0;
        }
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          dn[m] = sn[m] = 0.0f;
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = qb + m * stride;
          const float eq = ecell(q);
          dn[m] = (__ldcg(Z + q) + eq) + beta * __ldcg(dold + q);
          float s = 0.0f;
#pragma unroll
          for (int d = 0; d < 6; ++d)
            if (cd[m] & (1 << d)) {
              const int64_t nq = nb_index(q, d, a.nbr);
              if (GF_IN(nq, total)) {
                const float en = (nq >> 9) == (q >> 9) ? eq : ecell(nq);
                s = s + ((__ldcg(Z + nq) + en) + beta * __ldcg(dold + nq));
              }
            }
          sn[m] = s;
        }
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = qb + m * stride;
          const float diag = (float)((cd[m] >> CODE_DIAG_SHIFT) & 7);
          const float ad = diag * dn[m] - sn[m];
          dnew[q] = dn[m];
          AD[q] = ad;
          v[0] += (Acc)(dn[m] * ad);
        }
      }
      if (!grid_reduce<Acc, 1>(a, v, [&](double *t) {
            const double pAp = t[0];
            double al = (Acc)fabs(pAp) < (Acc)1.0e-30 ? 0.0 : (double)((Acc)st->rz / (Acc)pAp);
            if (!(pAp == pAp)) {  // NaN
              st->status = GF_NAN;
              st->done = 1;
            }
            st->alpha = al;
          }))
        return;
    }
    // ---- phase B: x += alpha d ; r -= alpha Ad ; z = M^-1 r ; r.z, r.r
    {
      const float alpha = (float)ld_volatile_d(&st->alpha);
      const float nalpha = -alpha;
      Acc v[2] = {0, 0};
      if (SGS) {
        const int tid = threadIdx.x;
        for (int base = blockIdx.x * SGS_TB; base < na; base += gridDim.x * SGS_TB) {
          uint16_t cd[SGS_TB];
          float dd[SGS_TB], xx[SGS_TB], rr[SGS_TB], aa[SGS_TB];
#pragma unroll
          for (int m = 0; m < SGS_TB; ++m) {
            const int64_t q = (int64_t)(base + m) * 512 + tid;
            cd[m] = base + m < na ? CODE[q] : (uint16_t)0;
            dd[m] = xx[m] = rr[m] = aa[m] = 0.0f;
            if (!(cd[m] & CODE_FLUID)) continue;
            dd[m] = __ldcg(dnew + q);
            xx[m] = __ldcg(X + q);
            rr[m] = __ldcg(R + q);
            aa[m] = __ldcg(AD + q);
          }
#pragma unroll
          for (int m = 0; m < SGS_TB; ++m) {
            const int64_t q = (int64_t)(base + m) * 512 + tid;
            float rn = 0.0f;
            if (cd[m] & CODE_FLUID) {
              X[q] = xx[m] + alpha * dd[m];
              rn = rr[m] + nalpha * aa[m];
              R[q] = rn;
            }
            rr[m] = rn;
            S.r[m * 512 + tid] = rn;
            S.code[m * 512 + tid] = cd[m];
            S.zb[m * 1000 + tile_pad(tid)] = rn * sgs_factor(cd[m]);
          }
          sgs_sweeps(S, a.sgs);
#pragma unroll
          for (int m = 0; m < SGS_TB; ++m) {
            if (!(cd[m] & CODE_FLUID)) continue;
            const int64_t q = (int64_t)(base + m) * 512 + tid;
            const float z = S.zb[m * 1000 + tile_pad(tid)];
            Z[q] = z;
            v[0] += (Acc)(rr[m] * z);
            v[1] += (Acc)(rr[m] * rr[m]);
          }
          if (coarse) tile_sums(base, rr);
          __syncthreads();
        }
      } else
      for (int64_t qb = q0; qb < total; qb += KQ * stride) {
        uint16_t cd[KQ];
        float dd[KQ], xx[KQ], rr[KQ], aa[KQ];
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          const int64_t q = qb + m * stride;
          cd[m] = q < total ? CODE[q] : (uint16_t)0;
        }
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          dd[m] = xx[m] = rr[m] = aa[m] = 0.0f;
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = qb + m * stride;
          dd[m] = __ldcg(dnew + q);
          xx[m] = __ldcg(X + q);
          rr[m] = __ldcg(R + q);
          aa[m] = __ldcg(AD + q);
        }
#pragma unroll
        for (int m = 0; m < KQ; ++m) {
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = qb + m * stride;
          X[q] = xx[m] + alpha * dd[m];
          const float rn = rr[m] + nalpha * aa[m];
          const float diag = fmaxf((float)((cd[m] >> CODE_DIAG_SHIFT) & 7), 1.0f);
          const float z = rn / diag;
          R[q] = rn;
          Z[q] = z;
          v[0] += (Acc)(rn * z);
          v[1] += (Acc)(rn * rn);
        }
      }
      const int it1 = it + 1;
      if (!grid_reduce<Acc, 2>(a, v, [&](double *t) {
            const double rz_new = t[0], rr = t[1];
            st->iters = it1;
            st->rr = rr;
            if (!(rr == rr)) {
              st->status = GF_NAN;
              st->done = 1;
              return;
            }
            int replace = 0;
            if (REF) {
              replace = rr < a.replace2 * st->r_upd2 || rr < a.tol2 * st->b2;
            } else {
              const bool check = (it1 % a.check_every) == 0 || it1 == a.max_iter;
              if (check && rr < a.tol2 * st->r0) st->done = 1;
            }
            if (replace) {
              st->n_replace = -st->n_replace - 1;  // negative: replacement pending
            } else if (coarse) {
              st->rz_part = rz_new;  // beta once the coarse term is in
            } else {
              const double rz = st->rz;
              st->beta = (Acc)fabs(rz) < (Acc)1.0e-30 ? 0.0 : (double)((Acc)rz_new / (Acc)rz);
              st->rz = rz_new;
            }
          }))
        return;
      // the coarse term of r . u and beta (not when a replacement recomputes r)
      if (coarse && !(REF && ld_volatile_i(&st->n_replace) < 0) && !ld_volatile_i(&st->done) &&
          !coarse_step([&](double *t) {
            const double rz = st->rz, rz_new = st->rz_part + t[0];
            st->beta = fabs(rz) < 1.0e-30 ? 0.0 : rz_new / rz;
            st->rz = rz_new;
          }))
        return;
    }
    // ---- refined: FP64 residual replacement r = b - A x
    if (REF && ld_volatile_i(&st->n_replace) < 0) {
      for (int64_t q = q0; q < total; q += stride) {
        if (!(a.code[q] & CODE_FLUID)) continue;
        a.x64[q] = __ldcg(a.x64 + q) + (double)__ldcg(a.x + q);
        a.x[q] = 0.0f;
      }
      if (!grid_barrier(a)) return;
      double v[3] = {0, 0, 0};
      auto residual = [&](int64_t q, uint16_t code) {  // b - A x64 in FP64
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < 6; ++d)
          if (code & (1 << d)) {
            const int64_t nq = nb_index(q, d, a.nbr);
            if (GF_IN(nq, total)) s += __ldcg(a.x64 + nq);
          }
        const double diag = (double)((code >> CODE_DIAG_SHIFT) & 7);
        return (double)(a.sign * a.bdiv[q]) - (diag * __ldcg(a.x64 + q) - s);
      };
      if (SGS) {
        const int tid = threadIdx.x;
        for (int base = blockIdx.x * SGS_TB; base < na; base += gridDim.x * SGS_TB) {
          float rf[SGS_TB];
#pragma unroll
          for (int m = 0; m < SGS_TB; ++m) {
            const int64_t q = (int64_t)(base + m) * 512 + tid;
            const uint16_t code = base + m < na ? CODE[q] : (uint16_t)0;
            rf[m] = 0.0f;
            if (code & CODE_FLUID) {
              const double res = residual(q, code);
              rf[m] = (float)res;
              a.r[q] = rf[m];
              v[0] += res * res;
            }
            S.r[m * 512 + tid] = rf[m];
            S.code[m * 512 + tid] = code;
            S.zb[m * 1000 + tile_pad(tid)] = rf[m] * sgs_factor(code);
          }
          sgs_sweeps(S, a.sgs);
#pragma unroll
          for (int m = 0; m < SGS_TB; ++m) {
            if (!(S.code[m * 512 + tid] & CODE_FLUID)) continue;
            const int64_t q = (int64_t)(base + m) * 512 + tid;
            const float z = S.zb[m * 1000 + tile_pad(tid)];
            a.z[q] = z;
            v[1] += (double)(rf[m] * z);
            v[2] += (double)(rf[m] * rf[m]);
          }
          if (coarse) tile_sums(base, rf);
          __syncthreads();
        }
      } else {
        for (int64_t q = q0; q < total; q += stride) {
          const uint16_t code = a.code[q];
          if (!(code & CODE_FLUID)) continue;
          const double res = residual(q, code);
          const float rf = (float)res;
          const float z = rf / fmaxf((float)((code >> CODE_DIAG_SHIFT) & 7), 1.0f);
          a.r[q] = rf;
          a.z[q] = z;
          v[0] += res * res;
          v[1] += (double)(rf * z);
          v[2] += (double)(rf * rf);
        }
      }
      if (!grid_reduce<double, 3>(a, v, [&](double *t) {
            st->r_true2 = t[0];
            st->r_upd2 = t[2];
            st->rr = t[2];
            st->n_replace = -st->n_replace;  // back to a positive count (+1)
            if (coarse) {
              st->rz_part = t[1];
            } else {
              const double rz = st->rz;
              st->beta = fabs(rz) < 1.0e-30 ? 0.0 : t[1] / rz;
              st->rz = t[1];
            }
            if (t[0] <= a.tol2 * st->b2) st->done = 1;
          }))
        return;
      if (coarse && !ld_volatile_i(&st->done) &&
          !coarse_step([&](double *t) {
            const double rz = st->rz, rz_new = st->rz_part + t[0];
            st->beta = fabs(rz) < 1.0e-30 ? 0.0 : rz_new / rz;
            st->rz = rz_new;
          }))
        return;
    }
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    if (!ld_volatile_i(&st->done)) st->status = GF_NOT_CONVERGED;
    st->coarse_used = coarse ? 1 : 0;
  }
}

// ------------------------------------------------------- segmented PCG
// The Jacobi-PCG of k_pcg for a batch of independent scenes in ONE persistent
// cooperative kernel with no grid-wide synchronisation.  A planning kernel
// (k_pcg_plan) splits the resident blocks among the scenes in proportion to
// their active tiles: a scene gets `nb` blocks of its own (rank 0..nb-1,
// tiles slot0[s] + rank + k*nb), and scenes smaller than one block's share
// are packed several to a block and solved one after the other, each entirely
// inside that block (block barriers only).  The blocks of a multi-block scene
// meet at a scene barrier whose last arrival sums the scene's per-block
// partials in rank order (deterministic) and updates the scene's scalars.
// Every scene thus iterates at its own pace and stops at its own tolerance;
// no scene waits for another.
struct PcgJob {
  int scene, rank, nb, pbase;  // pbase: first partial of the scene's blocks
};

struct SegPcgArgs {
  const int32_t *n_active, *nbr, *slot0;  // slot0[nseg+1]
  int nseg;
  const uint16_t *code;
  const float *bdiv;
  float *x, *r, *z, *d0, *d1, *Ad;
  double *x64;
  double *partials;  // [3][pstride], indexed by pbase + rank
  int64_t pstride;
  PcgState *st;      // [nseg]: scalars, convergence and the scene barrier
  PcgState *g;       // error flag of the solve
  const int32_t *blk_job0;  // [grid+1] first job of each block
  const PcgJob *jobs;
  int max_iter, check_every;
  double tol2, replace2;
  float sign;
  int sgs;           // tile-local symmetric Gauss-Seidel sweeps (0: Jacobi)
};

// Job table (one thread): `grid` blocks; the target tiles per block grows
// from total/grid until the multi-block scenes leave at least one block for
// the packed small ones.
__global__ void k_pcg_plan(const int32_t *__restrict__ slot0, int nseg, int grid,
                           PcgState *__restrict__ st, int32_t *__restrict__ blk_job0,
                           PcgJob *__restrict__ jobs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int total = slot0[nseg];
  int target = (total + grid - 1) / grid;
  if (target < 1) target = 1;
  for (;;) {
    int big = 0;
    for (int s = 0; s < nseg; ++s) {
      const int n = slot0[s + 1] - slot0[s];
      if (n > target) big += (n + target - 1) / target;
    }
    if (big < grid || target >= total) break;
    target += target / 16 + 1;
  }
  int b = 0, jb = 0, pb = 0;
  for (int s = 0; s < nseg; ++s) {  // scenes larger than one share: own blocks
    const int n = slot0[s + 1] - slot0[s];
    if (n <= target) continue;
    const int nb = (n + target - 1) / target;
    for (int r = 0; r < nb; ++r) {
      blk_job0[b++] = jb;
      jobs[jb++] = PcgJob{s, r, nb, pb};
    }
    pb += nb;
  }
  // the block receiving packed small scenes (after its own big scene when
  // every block holds one)
  int cur = b < grid ? b : grid - 1;
  if (b < grid) blk_job0[b] = jb;
  int load = 0;
  for (int s = 0; s < nseg; ++s) {
    const int n = slot0[s + 1] - slot0[s];
    if (n > target || n == 0) continue;
    if (load >= target && cur + 1 < grid) {
      ++cur;
      blk_job0[cur] = jb;
      load = 0;
    }
    jobs[jb++] = PcgJob{s, 0, 1, pb++};
    load += n;
  }
  for (int q = cur + 1; q <= grid; ++q) blk_job0[q] = jb;
  for (int s = 0; s < nseg; ++s) {  // scenes without fluid are solved already
    st[s] = PcgState{};
    if (slot0[s + 1] == slot0[s]) st[s].done = 1;
  }
}

constexpr int SEG_TG = 4;  // tiles per block step: loads of 4 tiles in flight per thread
static_assert(SEG_TG == SGS_TB && TILE_CELLS == PCG_THREADS,
              "the segmented PCG's tile groups are the preconditioner's rounds");

// Block sums of NV per-thread values added to tot[] (shared, by thread 0),
// once per phase (all of a block's tiles belong to one scene):
// per-warp shuffle trees, then warp 0 sums the 16 warp values of each row in
// a fixed order.
template <typename T, int NV>
__device__ __forceinline__ void block_acc(const T (&v)[NV], double *tot) {
  __shared__ T sh[NV][16];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    T x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k][wid] = x;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      T x = lane < 16 ? sh[k][lane] : (T)0;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) tot[k] += (double)x;
    }
  }
  __syncthreads();
}

// Scene reduction + barrier: tot[] (shared, this block's sums) becomes the
// scene's totals and fin(totals) runs once; afterwards every block of the
// scene sees the updated scene state.  Returns false on a barrier timeout.
template <int NV, typename Fin>
__device__ __forceinline__ bool scene_reduce(const SegPcgArgs &a, const PcgJob &j, double *tot, Fin fin) {
  __shared__ int s_ok;
  PcgState *S = a.st + j.scene;
  if (j.nb == 1) {
    if (threadIdx.x == 0) fin(tot);
    __syncthreads();
    return true;
  }
  if (threadIdx.x == 0) {
    s_ok = 1;
#pragma unroll
    for (int k = 0; k < NV; ++k) a.partials[k * a.pstride + j.pbase + j.rank] = tot[k];
    const unsigned gen = ld_volatile(&S->bar_gen);
    __threadfence();
    const unsigned arrived = atomicAdd(&S->bar_count, 1u);
    if (arrived == (unsigned)j.nb - 1) {
      __threadfence();
      double all[NV];
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        all[k] = 0.0;
        for (int r = 0; r < j.nb; ++r) all[k] += __ldcg(a.partials + k * a.pstride + j.pbase + r);
      }
      fin(all);
      __threadfence();
      atomicExch(&S->bar_count, 0u);
      __threadfence();
      atomicAdd(&S->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (ld_volatile(&S->bar_gen) == gen) {
        if (++spins > SPIN_LIMIT) {
          atomicExch(&a.g->error, 1);
          s_ok = 0;
          break;
        }
        __nanosleep(32);
      }
      __threadfence();
    }
  }
  __syncthreads();
  return s_ok && !ld_volatile_i(&a.g->error);
}

template <typename Acc, bool REF, bool SGS>
__device__ __forceinline__ bool pcg_scene(const SegPcgArgs &a, const PcgJob &j) {
  __shared__ double tot[3];
  // boxes of the tile preconditioner (SGS instantiation), rings zero throughout
  __shared__ alignas(16) unsigned char sg_raw[SGS ? sizeof(SgsSmem) : 16];
  SgsSmem &SG = *reinterpret_cast<SgsSmem *>(sg_raw);
  if (SGS) {
    for (int q = threadIdx.x; q < SGS_TB * 1000; q += blockDim.x) SG.zb[q] = 0.f;
    __syncthreads();
  }
  __shared__ float s_scal;   // alpha or beta of the running phase
  __shared__ int s_flag;     // done / replacement pending
  PcgState *S = a.st + j.scene;
  const int tid = threadIdx.x;
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;  // compact cells (bounds checks)
  (void)total;
  const int t_begin = __ldg(a.slot0 + j.scene) + j.rank, t_end = __ldg(a.slot0 + j.scene + 1);
  const int step = SEG_TG * j.nb;
  float *__restrict__ X = a.x;
  float *__restrict__ R = a.r;
  float *__restrict__ Z = a.z;
  float *__restrict__ AD = a.Ad;
  const uint16_t *__restrict__ CODE = a.code;
  auto clear = [&]() {
    if (tid < 3) tot[tid] = 0.0;
    __syncthreads();
  };
  // Each phase walks the block's tiles SEG_TG at a time and issues every load
  // of the group before any store, so the loads of the group's tiles are in
  // flight together.
  // ---- init: r = b, z = M^-1 r
  clear();
  {
    Acc v[2] = {0, 0};  // this thread's sums over all the block's tiles
    for (int base = t_begin; base < t_end; base += step) {
      uint16_t cd[SEG_TG];
      float bb[SEG_TG];
#pragma unroll
      for (int m = 0; m < SEG_TG; ++m) {
        const int sl = base + m * j.nb;
        const int64_t q = (int64_t)sl * TILE_CELLS + tid;
        cd[m] = sl < t_end ? CODE[q] : (uint16_t)0;
        bb[m] = (cd[m] & CODE_FLUID) ? a.bdiv[q] : 0.0f;
      }
      if (SGS) {  // z = M^-1 r by tile-local symmetric Gauss-Seidel sweeps
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          const float b = (cd[m] & CODE_FLUID) ? a.sign * bb[m] : 0.0f;
          if (cd[m] & CODE_FLUID) R[q] = b;
          bb[m] = b;
          SG.r[m * 512 + tid] = b;
          SG.code[m * 512 + tid] = cd[m];
          SG.zb[m * 1000 + tile_pad(tid)] = b * sgs_factor(cd[m]);
        }
        sgs_sweeps(SG, a.sgs);
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          const float z = SG.zb[m * 1000 + tile_pad(tid)];
          Z[q] = z;
          v[0] += (Acc)(bb[m] * z);
          v[1] += (Acc)(bb[m] * bb[m]);
        }
        __syncthreads();
        continue;
      }
#pragma unroll
      for (int m = 0; m < SEG_TG; ++m) {
        if (!(cd[m] & CODE_FLUID)) continue;
        const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
        const float b = a.sign * bb[m];
        const float diag = fmaxf((float)((cd[m] >> CODE_DIAG_SHIFT) & 7), 1.0f);
        const float z = b / diag;
        R[q] = b;
        Z[q] = z;
        v[0] += (Acc)(b * z);
        v[1] += (Acc)(b * b);
      }
    }
    block_acc<Acc, 2>(v, tot);
  }
  if (!scene_reduce<2>(a, j, tot, [&](double *t) {
        S->rz = t[0]; S->r0 = t[1]; S->rr = t[1]; S->b2 = t[1];
        S->r_upd2 = t[1]; S->r_true2 = t[1];
        S->beta = 0.0; S->alpha = 0.0; S->iters = 0; S->n_replace = 0; S->status = GF_OK;
        S->done = t[1] < 1e-30 ? 1 : 0;  // the reference's early exit (:2982-2986)
      }))
    return false;

  for (int it = 0; it < a.max_iter; ++it) {
    if (tid == 0) {
      s_flag = ld_volatile_i(&S->done);
      s_scal = (float)ld_volatile_d(&S->beta);
    }
    clear();
    if (s_flag) break;
    const float beta = s_scal;
    const float *__restrict__ dold = (it & 1) ? a.d1 : a.d0;
    float *__restrict__ dnew = (it & 1) ? a.d0 : a.d1;
    // ---- phase A: d = z + beta d ; Ad = A d ; d.Ad
    {
      Acc v[1] = {0};
      for (int base = t_begin; base < t_end; base += step) {
        uint16_t cd[SEG_TG];
        float dn[SEG_TG], sn[SEG_TG];
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          const int sl = base + m * j.nb;
          const int64_t q = (int64_t)sl * TILE_CELLS + tid;
          cd[m] = sl < t_end ? CODE[q] : (uint16_t)0;
        }
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          dn[m] = 0.0f;
          sn[m] = 0.0f;
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          dn[m] = __ldcg(Z + q) + beta * __ldcg(dold + q);
          float s = 0.0f;
#pragma unroll
          for (int d = 0; d < 6; ++d)
            if (cd[m] & (1 << d)) {
              const int64_t nq = nb_index(q, d, a.nbr);
              if (GF_IN(nq, total)) s = s + (__ldcg(Z + nq) + beta * __ldcg(dold + nq));
            }
          sn[m] = s;
        }
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          const float diag = (float)((cd[m] >> CODE_DIAG_SHIFT) & 7);
          const float ad = diag * dn[m] - sn[m];
          dnew[q] = dn[m];
          AD[q] = ad;
          v[0] += (Acc)(dn[m] * ad);
        }
      }
      block_acc<Acc, 1>(v, tot);
    }
    if (!scene_reduce<1>(a, j, tot, [&](double *t) {
          const double pAp = t[0];
          S->alpha = (Acc)fabs(pAp) < (Acc)1.0e-30 ? 0.0 : (double)((Acc)S->rz / (Acc)pAp);
          if (!(pAp == pAp)) {
            S->status = GF_NAN;
            S->done = 1;
          }
        }))
      return false;
    if (tid == 0) {
      s_flag = ld_volatile_i(&S->done);
      s_scal = (float)ld_volatile_d(&S->alpha);
    }
    clear();
    if (s_flag) break;
    // ---- phase B: x += alpha d ; r -= alpha Ad ; z = M^-1 r ; r.z, r.r
    {
      const float alpha = s_scal;
      const float nalpha = -alpha;
      Acc v[2] = {0, 0};
      for (int base = t_begin; base < t_end; base += step) {
        uint16_t cd[SEG_TG];
        float dd[SEG_TG], xx[SEG_TG], rr[SEG_TG], aa[SEG_TG];
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          const int sl = base + m * j.nb;
          const int64_t q = (int64_t)sl * TILE_CELLS + tid;
          cd[m] = sl < t_end ? CODE[q] : (uint16_t)0;
        }
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          dd[m] = xx[m] = rr[m] = aa[m] = 0.0f;
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          dd[m] = __ldcg(dnew + q);
          xx[m] = __ldcg(X + q);
          rr[m] = __ldcg(R + q);
          aa[m] = __ldcg(AD + q);
        }
        if (SGS) {
#pragma unroll
          for (int m = 0; m < SEG_TG; ++m) {
            const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
            float rn = 0.0f;
            if (cd[m] & CODE_FLUID) {
              X[q] = xx[m] + alpha * dd[m];
              rn = rr[m] + nalpha * aa[m];
              R[q] = rn;
            }
            rr[m] = rn;
            SG.r[m * 512 + tid] = rn;
            SG.code[m * 512 + tid] = cd[m];
            SG.zb[m * 1000 + tile_pad(tid)] = rn * sgs_factor(cd[m]);
          }
          sgs_sweeps(SG, a.sgs);
#pragma unroll
          for (int m = 0; m < SEG_TG; ++m) {
            if (!(cd[m] & CODE_FLUID)) continue;
            const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
            const float z = SG.zb[m * 1000 + tile_pad(tid)];
            Z[q] = z;
            v[0] += (Acc)(rr[m] * z);
            v[1] += (Acc)(rr[m] * rr[m]);
          }
          __syncthreads();
          continue;
        }
#pragma unroll
        for (int m = 0; m < SEG_TG; ++m) {
          if (!(cd[m] & CODE_FLUID)) continue;
          const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
          X[q] = xx[m] + alpha * dd[m];
          const float rn = rr[m] + nalpha * aa[m];
          const float diag = fmaxf((float)((cd[m] >> CODE_DIAG_SHIFT) & 7), 1.0f);
          const float z = rn / diag;
          R[q] = rn;
          Z[q] = z;
          v[0] += (Acc)(rn * z);
          v[1] += (Acc)(rn * rn);
        }
      }
      block_acc<Acc, 2>(v, tot);
    }
    const int it1 = it + 1;
    if (!scene_reduce<2>(a, j, tot, [&](double *t) {
          const double rz_new = t[0], rr = t[1];
          S->iters = it1;
          S->rr = rr;
          if (!(rr == rr)) {
            S->status = GF_NAN;
            S->done = 1;
            return;
          }
          int replace = 0;
          if (REF) {
            replace = rr < a.replace2 * S->r_upd2 || rr < a.tol2 * S->b2;
          } else {
            const bool check = (it1 % a.check_every) == 0 || it1 == a.max_iter;
            if (check && rr < a.tol2 * S->r0) S->done = 1;
          }
          if (replace) {
            S->n_replace = -S->n_replace - 1;  // negative: replacement pending
          } else {
            const double rz = S->rz;
            S->beta = (Acc)fabs(rz) < (Acc)1.0e-30 ? 0.0 : (double)((Acc)rz_new / (Acc)rz);
            S->rz = rz_new;
          }
        }))
      return false;
    // ---- refined: FP64 residual replacement r = b - A x
    if (REF) {
      if (tid == 0) s_flag = ld_volatile_i(&S->n_replace) < 0;
      clear();
      if (s_flag) {
        for (int sl = t_begin; sl < t_end; sl += j.nb) {
          const int64_t q = (int64_t)sl * TILE_CELLS + tid;
          if (!(CODE[q] & CODE_FLUID)) continue;
          a.x64[q] = __ldcg(a.x64 + q) + (double)__ldcg(X + q);
          X[q] = 0.0f;
        }
        __syncthreads();
        if (!scene_reduce<1>(a, j, tot, [](double *) {})) return false;  // x64 complete
        double v[3] = {0, 0, 0};
        for (int base = t_begin; base < t_end; base += step) {
          uint16_t cd[SEG_TG];
          double res[SEG_TG];
#pragma unroll
          for (int m = 0; m < SEG_TG; ++m) {
            const int sl = base + m * j.nb;
            const int64_t q = (int64_t)sl * TILE_CELLS + tid;
            cd[m] = sl < t_end ? CODE[q] : (uint16_t)0;
          }
#pragma unroll
          for (int m = 0; m < SEG_TG; ++m) {
            res[m] = 0.0;
            if (!(cd[m] & CODE_FLUID)) continue;
            const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
            double s = 0.0;
#pragma unroll
            for (int d = 0; d < 6; ++d)
              if (cd[m] & (1 << d)) {
                const int64_t nq = nb_index(q, d, a.nbr);
                if (GF_IN(nq, total)) s += __ldcg(a.x64 + nq);
              }
            const double diag = (double)((cd[m] >> CODE_DIAG_SHIFT) & 7);
            res[m] = (double)(a.sign * a.bdiv[q]) - (diag * __ldcg(a.x64 + q) - s);
          }
          if (SGS) {
            float rf[SEG_TG];
#pragma unroll
            for (int m = 0; m < SEG_TG; ++m) {
              const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
              rf[m] = (cd[m] & CODE_FLUID) ? (float)res[m] : 0.0f;
              if (cd[m] & CODE_FLUID) {
                R[q] = rf[m];
                v[0] += res[m] * res[m];
              }
              SG.r[m * 512 + tid] = rf[m];
              SG.code[m * 512 + tid] = cd[m];
              SG.zb[m * 1000 + tile_pad(tid)] = rf[m] * sgs_factor(cd[m]);
            }
            sgs_sweeps(SG, a.sgs);
#pragma unroll
            for (int m = 0; m < SEG_TG; ++m) {
              if (!(cd[m] & CODE_FLUID)) continue;
              const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
              const float z = SG.zb[m * 1000 + tile_pad(tid)];
              Z[q] = z;
              v[1] += (double)(rf[m] * z);
              v[2] += (double)(rf[m] * rf[m]);
            }
            __syncthreads();
            continue;
          }
#pragma unroll
          for (int m = 0; m < SEG_TG; ++m) {
            if (!(cd[m] & CODE_FLUID)) continue;
            const int64_t q = (int64_t)(base + m * j.nb) * TILE_CELLS + tid;
            const float rf = (float)res[m];
            const float diag = fmaxf((float)((cd[m] >> CODE_DIAG_SHIFT) & 7), 1.0f);
            const float z = rf / diag;
            R[q] = rf;
            Z[q] = z;
            v[0] += res[m] * res[m];
            v[1] += (double)(rf * z);
            v[2] += (double)(rf * rf);
          }
        }
        block_acc<double, 3>(v, tot);
        if (!scene_reduce<3>(a, j, tot, [&](double *t) {
              S->r_true2 = t[0];
              S->r_upd2 = t[2];
              S->rr = t[2];
              S->n_replace = -S->n_replace;  // back to a positive count (+1)
              const double rz = S->rz;
              S->beta = fabs(rz) < 1.0e-30 ? 0.0 : t[1] / rz;
              S->rz = t[1];
              if (t[0] <= a.tol2 * S->b2) S->done = 1;
            }))
          return false;
      }
    }
  }
  if (tid == 0 && j.rank == 0 && !ld_volatile_i(&S->done)) S->status = GF_NOT_CONVERGED;
  return true;
}

template <typename Acc, bool REF, bool SGS>
__global__ void __launch_bounds__(TILE_CELLS, 2) k_pcg_seg(SegPcgArgs a) {
  const int j0 = a.blk_job0[blockIdx.x], j1 = a.blk_job0[blockIdx.x + 1];
  for (int jj = j0; jj < j1; ++jj) {
    const PcgJob j = a.jobs[jj];
    if (ld_volatile_i(&a.st[j.scene].done)) continue;  // no fluid
    if (!pcg_scene<Acc, REF, SGS>(a, j)) return;
  }
}

struct ScatterArgs {
  const int32_t *n_active, *tile_list;
  const uint16_t *code;
  const float *x;
  const double *x64;
  float *p;
  int ny, nz, nty, ntz;
  // solve health: the statuses of the solve just finished (nst scenes,
  // nullptr for the fixed-sweep Jacobi / GS-RB), the solve's barrier-timeout
  // flag, and the context's health words
  const PcgState *st;
  const PcgState *st_err;
  int nst;
  int32_t *health;
  int64_t ncell;  // cells of p (all scenes of a batch)
};

// Severity of a solve status: OK < NOT_CONVERGED < BREAKDOWN < NAN < TIMEOUT.
__host__ __device__ inline int status_severity(int s) {
  switch (s) {
    case GF_OK: return 0;
    case GF_NOT_CONVERGED: return 1;
    case GF_BREAKDOWN: return 2;
    case GF_NAN: return 3;
    case GF_TIMEOUT: return 4;
    default: return 2;
  }
}

// Block 0 folds the finished solve into the context's health words: one
// solve per scene, the worst severity since the last reset and of this call,
// and the counts of solves that stopped at their cap or failed.  Runs before
// the scatter loop, uniformly in block 0 (it holds a block barrier).
__device__ void fold_health(const ScatterArgs &a) {
  if (blockIdx.x != 0 || a.health == nullptr) return;
  __shared__ int s_worst;
  if (threadIdx.x == 0) s_worst = 0;
  __syncthreads();
  const bool timeout = a.st_err != nullptr && ld_volatile_i(&a.st_err->error) != 0;
  int nc = 0, nfail = 0, worst = 0;
  for (int s = threadIdx.x; s < a.nst; s += blockDim.x) {
    const int status = a.st == nullptr ? GF_OK : (timeout ? GF_TIMEOUT : a.st[s].status);
    const int sev = status_severity(status);
    worst = sev > worst ? sev : worst;
    nc += status == GF_NOT_CONVERGED;
    nfail += sev >= 2;
  }
  if (worst) atomicMax(&s_worst, worst);
  if (nc) atomicAdd(&a.health[2], nc);
  if (nfail) atomicAdd(&a.health[3], nfail);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&a.health[0], s_worst);
    atomicAdd(&a.health[1], a.nst);
    a.health[4] = s_worst;
  }
}

__global__ void k_scatter_p(ScatterArgs a) {
  fold_health(a);
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    if (!(a.code[q] & CODE_FLUID)) continue;
    const int s = (int)(q >> 9), l = (int)(q & 511);
    const int t = a.tile_list[s];
    const int ti = t / (a.nty * a.ntz), tj = (t / a.ntz) % a.nty, tk = t % a.ntz;
    const int gi = ti * 8 + (l >> 6), gj = tj * 8 + ((l >> 3) & 7), gk = tk * 8 + (l & 7);
    float v = a.x[q];
    if (a.x64) v = (float)(a.x64[q] + (double)v);
    const int64_t g = ((int64_t)gi * a.ny + gj) * a.nz + gk;
    if (GF_IN(g, a.ncell)) a.p[g] = v;
  }
}

__global__ void kb_scatter_p(ScatterArgs a, SegIndex sx) {
  fold_health(a);
  const int64_t total = (int64_t)(*a.n_active) * TILE_CELLS;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    if (!(a.code[q] & CODE_FLUID)) continue;
    const int s = (int)(q >> 9), l = (int)(q & 511);
    const int tg = a.tile_list[s];
    const SegRow r = sx.row[seg_find(sx.tile0, sx.n, tg)];
    const int t = (int)(tg - r.tile0);
    const int ti = t / (r.nty * r.ntz), tj = (t / r.ntz) % r.nty, tk = t % r.ntz;
    const int gi = ti * 8 + (l >> 6), gj = tj * 8 + ((l >> 3) & 7), gk = tk * 8 + (l & 7);
    float v = a.x[q];
    if (a.x64) v = (float)(a.x64[q] + (double)v);
    const int64_t g = r.cell0 + ((int64_t)gi * r.ny + gj) * r.nz + gk;
    if (GF_IN(g, a.ncell)) a.p[g] = v;
  }
}

// ------------------------------------------------------------- host side
int pressure_alloc(Ctx *c) {
  const int64_t nk = c->nkeys;
  auto A = [&](void **p, size_t bytes, const char *what) {
    return check_cuda(c, cudaMalloc(p, bytes), what);
  };
  int e;
  if ((e = A((void **)&c->tile_slot, c->ntiles * 4, "alloc tile_slot"))) return e;
  if ((e = A((void **)&c->tile_list, c->ntiles * 4, "alloc tile_list"))) return e;
  if (c->nseg == 0) {  // Morton order of the tile grid for the slot numbering
    std::vector<std::pair<uint64_t, int32_t>> key(c->ntiles);
    auto spread = [](uint64_t v) {  // bits of v at every third position
      uint64_t r = 0;
      for (int b = 0; b < 21; ++b) r |= ((v >> b) & 1ull) << (3 * b);
      return r;
    };
    for (int t = 0; t < c->ntiles; ++t) {
      const int ti = t / (c->nty * c->ntz), tj = (t / c->ntz) % c->nty, tk = t % c->ntz;
      key[t] = {(spread(ti) << 2) | (spread(tj) << 1) | spread(tk), t};
    }
    std::sort(key.begin(), key.end());
    std::vector<int32_t> ord(c->ntiles);
    for (int t = 0; t < c->ntiles; ++t) ord[t] = key[t].second;
    if ((e = A((void **)&c->tile_order, c->ntiles * 4, "alloc tile_order"))) return e;
    if ((e = check_cuda(c, cudaMemcpy(c->tile_order, ord.data(), c->ntiles * 4,
                                      cudaMemcpyHostToDevice), "upload tile_order")))
      return e;
  }
  if ((e = A((void **)&c->tile_nbr, (size_t)c->ntiles * 6 * 4, "alloc tile_nbr"))) return e;
  if ((e = A((void **)&c->n_active, 16, "alloc n_active"))) return e;
  if ((e = A((void **)&c->code, nk * 2, "alloc code"))) return e;
  float **vecs[7] = {&c->bdiv, &c->xf, &c->r, &c->z, &c->d0, &c->d1, &c->Ad};
  for (int q = 0; q < 7; ++q)
    if ((e = A((void **)vecs[q], nk * 4, "alloc pressure vector"))) return e;
  if ((e = A((void **)&c->x64, nk * 8, "alloc x64"))) return e;
  // per-block partials of the PCGs; a batch's segmented PCG indexes them by
  // job (at most one per scene plus one per block)
  const int64_t np = (int64_t)c->ntiles + MAX_PCG_BLOCKS;
  if ((e = A((void **)&c->partials, 3 * np * sizeof(double), "alloc partials"))) return e;
  if ((e = A((void **)&c->state, sizeof(PcgState), "alloc pcg state"))) return e;
  if ((e = A((void **)&c->bar_counters, BAR_BYTES, "alloc barrier counters"))) return e;
  if ((e = A((void **)&c->trace, TRACE_CAP * 8, "alloc trace"))) return e;
  if ((e = A((void **)&c->halo, nk * 6 * 4, "alloc halo buffers"))) return e;
  // coarse operator and its inverse (GF_FLAG_COARSE), allocated up front so
  // that solves can be captured in CUDA graphs
  if ((e = A((void **)&c->coarse_buf, (size_t)COARSE_BUF_BYTES, "alloc coarse operator")))
    return e;
  // the cube regions of the global-memory solver: the smallest power-of-two
  // edge (in tiles) that keeps the region grid within COARSE_RG_DENSE_MAX
  {
    RegionGrid &g = c->rg;
    g.ntx = c->ntx;
    g.nty = c->nty;
    g.ntz = c->ntz;
    g.ct = 1;
    for (;;) {
      g.nx = (g.ntx + g.ct - 1) / g.ct;
      g.ny = (g.nty + g.ct - 1) / g.ct;
      g.nz = (g.ntz + g.ct - 1) / g.ct;
      g.n = g.nx * g.ny * g.nz;
      if (g.n <= COARSE_RG_DENSE_MAX) break;
      g.ct *= 2;
    }
  }
  const int64_t nids = c->ntiles > c->rg.n ? c->ntiles : c->rg.n;
  if ((e = A((void **)&c->coarse_prev_slot, (size_t)nids * 4, "alloc coarse row map"))) return e;
  // no B yet: meta zero, no id has a row
  if ((e = check_cuda(c, cudaMemset(c->coarse_buf + COARSE_META_OFF, 0, sizeof(CoarseMeta)),
                      "zero coarse meta")) ||
      (e = check_cuda(c, cudaMemset(c->coarse_prev_slot, 0xff, (size_t)nids * 4),
                      "clear coarse row map")))
    return e;
  {
    const RegionGrid &g = c->rg;
    const int64_t ni = 2 * (int64_t)g.n + COARSE_RMAX + 4 + (int64_t)COARSE_RMAX * 6 +
                       (int64_t)COARSE_RMAX * g.ct * g.ct * g.ct + c->ntiles;
    if ((e = A((void **)&c->rg_buf, (size_t)ni * 4, "alloc coarse regions")) ||
        (e = check_cuda(c, cudaMemset(c->rg_buf, 0, (size_t)g.n * 4), "zero region flags")) ||
        (e = A((void **)&c->rg_gt, (size_t)c->ntiles * 4, "alloc tile residual sums")) ||
        (e = A((void **)&c->rg_e, (size_t)COARSE_RMAX * 4, "alloc region corrections")))
      return e;
  }
  if ((e = A((void **)&c->tile_cost, (size_t)c->ntiles * 4, "alloc tile cost"))) return e;
  if ((e = A((void **)&c->health, 8 * 4, "alloc solve health"))) return e;
  if ((e = check_cuda(c, cudaMemset(c->health, 0, 8 * 4), "zero solve health"))) return e;
  if ((e = check_cuda(c, cudaMemset(c->state, 0, sizeof(PcgState)), "zero pcg state"))) return e;
  if ((e = check_cuda(c, cudaMallocHost((void **)&c->state_host, sizeof(PcgState)),
                      "alloc pinned state")))
    return e;
  memset(c->state_host, 0, sizeof(PcgState));
  return GF_OK;
}

void pressure_free(Ctx *c) {
  void *ps[] = {c->tile_slot, c->tile_list, c->tile_order, c->tile_nbr, c->n_active, c->code, c->bdiv,
                c->xf, c->r, c->z, c->d0, c->d1, c->Ad, c->x64, c->partials, c->state,
                c->bar_counters, c->trace, c->halo, c->tile_cost, c->coarse_buf,
                c->coarse_prev_slot, c->rg_buf, c->rg_gt, c->rg_e, c->health};
  for (void *p : ps)
    if (p) cudaFree(p);
  if (c->state_host) cudaFreeHost(c->state_host);
}

template <typename Acc, bool REF, bool SGS>
static int coop_grid(Ctx *c) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg<Acc, REF, SGS>,
                                                                PCG_THREADS, 0);
  if (e != cudaSuccess || per_sm < 1) return 0;
  if (c->tune.pcg_blocks_per_sm > 0 && c->tune.pcg_blocks_per_sm < per_sm)
    per_sm = c->tune.pcg_blocks_per_sm;
  int g = per_sm * c->num_sms;
  return g > MAX_PCG_BLOCKS ? MAX_PCG_BLOCKS : g;
}

template <typename Acc, bool REF, bool SGS>
static int launch_pcg_t(Ctx *c, PcgArgs &pa) {
  int g = coop_grid<Acc, REF, SGS>(c);
  if (g < 1) return fail(c, GF_CUDA_ERROR, "PCG: cooperative occupancy query failed");
  void *args[] = {&pa};
  int e = check_cuda(c, cudaLaunchCooperativeKernel((const void *)k_pcg<Acc, REF, SGS>, dim3(g),
                                                    dim3(PCG_THREADS), args, 0, c->stream),
                     "cooperative PCG launch");
  c->launches++;
  return e;
}

template <typename Acc, bool REF>
static int launch_pcg(Ctx *c, PcgArgs &pa) {
  return pa.sgs > 0 ? launch_pcg_t<Acc, REF, true>(c, pa) : launch_pcg_t<Acc, REF, false>(c, pa);
}

template <typename Acc, bool REF, bool SGS>
static int launch_pcg_seg_t(Ctx *c, SegPcgArgs &pa) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_seg<Acc, REF, SGS>,
                                                    TILE_CELLS, 0) != cudaSuccess ||
      per_sm < 1)
    return fail(c, GF_CUDA_ERROR, "segmented PCG: cooperative occupancy query failed");
  if (c->tune.pcg_blocks_per_sm > 0 && c->tune.pcg_blocks_per_sm < per_sm)
    per_sm = c->tune.pcg_blocks_per_sm;
  int grid = per_sm * c->num_sms;
  if (grid > MAX_PCG_BLOCKS) grid = MAX_PCG_BLOCKS;
  k_pcg_plan<<<1, 32, 0, c->stream>>>(c->seg_slot0, c->nseg, grid, c->seg_state,
                                      c->pcg_blk_job0, reinterpret_cast<PcgJob *>(c->pcg_jobs));
  c->launches++;
  pa.blk_job0 = c->pcg_blk_job0;
  pa.jobs = reinterpret_cast<const PcgJob *>(c->pcg_jobs);
  void *args[] = {&pa};
  int e = check_cuda(c, cudaLaunchCooperativeKernel((const void *)k_pcg_seg<Acc, REF, SGS>,
                                                    dim3(grid), dim3(TILE_CELLS), args, 0,
                                                    c->stream),
                     "cooperative segmented PCG launch");
  c->launches++;
  return e;
}

template <typename Acc, bool REF>
static int launch_pcg_seg(Ctx *c, SegPcgArgs &pa) {
  return pa.sgs > 0 ? launch_pcg_seg_t<Acc, REF, true>(c, pa)
                    : launch_pcg_seg_t<Acc, REF, false>(c, pa);
}

// Bytes of the job table of a batch with nseg scenes.
size_t pcg_jobs_bytes(int nseg) { return (size_t)(nseg + MAX_PCG_BLOCKS) * sizeof(PcgJob); }

// The pressure stage of a batch: set-up over every scene's tiles, then the
// sweeps (scene-agnostic on the compact layout) or the segmented PCG.
static int launch_pressure_batch(Ctx *c, const gf_step_params *prm) {
  cudaStream_t st = c->stream;
  const int solver = prm->solver;
  const SegIndex sx = seg_index(c);
  int e;
  int32_t *flag = c->tile_nbr;  // consumed by the compaction before the set-up
  kb_tile_flags<<<(unsigned)((c->ntiles * 32 + 255) / 256), 256, 0, st>>>(c->f.label, sx,
                                                                          c->ntiles, flag);
  k_tile_compact<<<1, 1024, 0, st>>>(flag, c->ntiles, nullptr, c->tile_slot, c->tile_list,
                                     c->n_active);
  kb_slot_ranges<<<(unsigned)((c->nseg + 256) / 256), 256, 0, st>>>(c->tile_list, c->n_active,
                                                                    sx, c->seg_slot0);
  c->launches += 3;
  const bool refined = solver == GF_PCG_REFINED;
  int64_t *n_fluid = reinterpret_cast<int64_t *>(c->n_active + 2);
  if ((e = check_cuda(c, cudaMemsetAsync(n_fluid, 0, 8, st), "zero fluid count"))) return e;
  BatchSetupArgs ba{{c->f.label, c->f.div, c->n_active, c->tile_list, c->tile_slot, c->tile_nbr,
                     c->code, c->bdiv, c->xf, c->r, c->z, c->d0, c->d1, c->Ad,
                     refined ? c->x64 : nullptr, n_fluid, c->tile_cost, 0, 0, 0, 0, 0, 0},
                    sx};
  {
    int g = c->ntiles < c->num_sms * 4 ? c->ntiles : c->num_sms * 4;
    kb_tile_setup<<<g > 0 ? g : 1, 512, 0, st>>>(ba);
    c->launches++;
  }
  const unsigned gs = (unsigned)(c->num_sms * 8);
  SweepArgs sw{c->n_active, c->tile_nbr, c->code, c->bdiv};
  const float *result = c->xf;
  const double *result64 = nullptr;
  if (c->timing) cudaEventRecord(c->ev[8], st);
  if (solver == GF_JACOBI) {
    float *a = c->xf, *b = c->z;
    for (int it = 0; it < prm->max_iters; ++it) {
      k_jacobi<<<gs, 256, 0, st>>>(sw, a, b);
      float *t = a; a = b; b = t;
    }
    c->launches += prm->max_iters;
    result = a;
    c->last_iters = prm->max_iters;
  } else if (solver == GF_GSRB) {
    for (int it = 0; it < prm->max_iters; ++it) {
      k_gsrb<<<gs, 256, 0, st>>>(sw, c->xf, 0);
      k_gsrb<<<gs, 256, 0, st>>>(sw, c->xf, 1);
    }
    c->launches += 2 * prm->max_iters;
    c->last_iters = prm->max_iters;
  } else {
    if ((e = check_cuda(c, cudaMemsetAsync(c->state, 0, sizeof(PcgState), st), "zero state")))
      return e;
    const int check_every = prm->check_every > 0 ? prm->check_every : 1;
    const float sign = prm->rhs_sign >= 0 ? 1.0f : -1.0f;
    SegPcgArgs pa{c->n_active, c->tile_nbr, c->seg_slot0, c->nseg, c->code, c->bdiv, c->xf,
                  c->r, c->z, c->d0, c->d1, c->Ad, refined ? c->x64 : nullptr, c->partials,
                  (int64_t)c->ntiles + MAX_PCG_BLOCKS, c->seg_state, c->state, nullptr,
                  nullptr, prm->max_iters, check_every, prm->tol * prm->tol, PCG_REPLACE2, sign,
                  (prm->flags & GF_FLAG_SGS_MASK) >> GF_FLAG_SGS_SHIFT};
    if (refined) {
      e = launch_pcg_seg<double, true>(c, pa);
      result64 = c->x64;
    } else {
      e = launch_pcg_seg<float, false>(c, pa);
    }
    if (e) return e;
  }
  if (c->timing) cudaEventRecord(c->ev[9], st);
  if ((e = check_cuda(c, cudaMemsetAsync(c->f.p, 0, c->ncell * 4, st), "zero p"))) return e;
  const bool pcg = solver == GF_PCG || solver == GF_PCG_REFINED;
  ScatterArgs sc{c->n_active, c->tile_list, c->code, result, result64, c->f.p, 0, 0, 0, 0,
                 pcg ? c->seg_state : nullptr, pcg ? c->state : nullptr, c->nseg, c->health,
                 c->ncell};
  kb_scatter_p<<<gs, 256, 0, st>>>(sc, sx);
  c->launches++;
  c->last_solver = solver;
  return check_launch(c, "gf_pressure");
}

int launch_pressure(Ctx *c, const gf_step_params *prm) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_pressure: buffers not bound");
  const int solver = prm->solver;
  if (solver < GF_JACOBI || solver > GF_PCG_REFINED)
    return fail(c, GF_INVALID_ARG, "unknown pressure_solver");
  if (prm->max_iters < 0) return fail(c, GF_INVALID_ARG, "pressure_iters must be >= 0");
  if (c->nseg > 0) return launch_pressure_batch(c, prm);
  cudaStream_t st = c->stream;
  int e;
  // ---- active tiles
  {
    // the flags live in tile_nbr (>= ntiles entries): k_tile_compact consumes
    // them before k_tile_setup overwrites that array with the neighbour table
    int32_t *flag = c->tile_nbr;
    unsigned g = (unsigned)((c->ntiles * 32 + 255) / 256);
    k_tile_flags<<<g, 256, 0, st>>>(c->f.label, c->nx, c->ny, c->nz, c->nty, c->ntz,
                                    c->ntiles, flag);
    k_tile_compact<<<1, 1024, 0, st>>>(flag, c->ntiles, c->tile_order, c->tile_slot, c->tile_list,
                                       c->n_active);
    c->launches += 2;
  }
  const bool refined = solver == GF_PCG_REFINED;
  int64_t *n_fluid = reinterpret_cast<int64_t *>(c->n_active + 2);
  if ((e = check_cuda(c, cudaMemsetAsync(n_fluid, 0, 8, st), "zero fluid count"))) return e;
  SetupArgs sa{c->f.label, c->f.div, c->n_active, c->tile_list, c->tile_slot, c->tile_nbr,
               c->code, c->bdiv, c->xf, c->r, c->z, c->d0, c->d1, c->Ad,
               refined ? c->x64 : nullptr, n_fluid, c->tile_cost, c->nx, c->ny, c->nz, c->ntx,
               c->nty, c->ntz};
  {
    int g = c->ntiles < c->num_sms * 4 ? c->ntiles : c->num_sms * 4;
    k_tile_setup<<<g > 0 ? g : 1, 512, 0, st>>>(sa);
    c->launches++;
  }
  const unsigned gs = (unsigned)(c->num_sms * 8);
  SweepArgs sw{c->n_active, c->tile_nbr, c->code, c->bdiv};
  const float *result = c->xf;
  const double *result64 = nullptr;
  if (c->timing) cudaEventRecord(c->ev[8], st);
  if (solver == GF_JACOBI) {
    float *a = c->xf, *b = c->z;
    for (int it = 0; it < prm->max_iters; ++it) {
      k_jacobi<<<gs, 256, 0, st>>>(sw, a, b);
      float *t = a; a = b; b = t;
    }
    c->launches += prm->max_iters;
    result = a;
    c->last_iters = prm->max_iters;
  } else if (solver == GF_GSRB) {
    for (int it = 0; it < prm->max_iters; ++it) {
      k_gsrb<<<gs, 256, 0, st>>>(sw, c->xf, 0);
      k_gsrb<<<gs, 256, 0, st>>>(sw, c->xf, 1);
    }
    c->launches += 2 * prm->max_iters;
    c->last_iters = prm->max_iters;
  } else {
    if ((e = check_cuda(c, cudaMemsetAsync(c->state, 0, sizeof(PcgState), st), "zero state")))
      return e;
    const int check_every = prm->check_every > 0 ? prm->check_every : 1;
    const float sign = prm->rhs_sign >= 0 ? 1.0f : -1.0f;
    const double replace2 = PCG_REPLACE2;
    const bool force_global =
        (prm->flags & GF_FLAG_GLOBAL_PCG) != 0 || !pcg_smem_fits(c, refined);
    if (!force_global) {
      if ((e = check_cuda(c, cudaMemsetAsync(c->bar_counters, 0, BAR_BYTES, st),
                          "zero barrier counters")))
        return e;
      // the one-round-trip reduction words of the shared-memory solver
      // ([2][160][4] u64 at 2048 doubles into the partials buffer), then the
      // tagged coarse sums ([2][COARSE_RMAX] u64)
      if ((e = check_cuda(c, cudaMemsetAsync(c->partials + 2048, 0,
                                             (2 * 160 * 4 + 2 * COARSE_RMAX) * 8, st),
                          "zero reduction words")))
        return e;
      const bool coarse = (prm->flags & GF_FLAG_COARSE) != 0;
      float *h = c->halo;
      const int64_t nk = c->nkeys;
      PcgSmemArgs sa{c->n_active, c->tile_nbr, c->tile_cost, c->code, c->bdiv, c->xf, h, h + nk, h + 2 * nk,
                     h + 3 * nk, h + 4 * nk, h + 5 * nk, refined ? c->x64 : nullptr,
                     c->partials, c->bar_counters, c->state,
                     (prm->flags & GF_FLAG_TRACE) ? c->trace : nullptr, TRACE_CAP,
                     prm->max_iters, check_every, prm->tol * prm->tol, replace2, sign,
                     (prm->flags & GF_FLAG_SGS_MASK) >> GF_FLAG_SGS_SHIFT,
                     coarse ? 1 : 0, c->coarse_buf,
                     (prm->flags & GF_FLAG_TEST_STALL) ? 1 : 0,
                     (refined && (prm->flags & GF_FLAG_WARM_START)) ? 1 : 0, c->f.p,
                     c->tile_list, c->ny, c->nz, c->nty, c->ntz};
      // the solver publishes tagged 64-bit halo words over the first two halo
      // arrays; their counts restart at 1 with every solve
      if ((e = check_cuda(c, cudaMemsetAsync(h, 0, (size_t)nk * 8, st), "zero tagged halo")))
        return e;
      if ((e = launch_pcg_smem(c, sa, refined))) return e;
    }
    PcgArgs pa{c->n_active, c->tile_nbr, c->code, c->bdiv, c->xf, c->r, c->z, c->d0, c->d1,
               c->Ad, refined ? c->x64 : nullptr, c->partials, c->state,
               prm->max_iters, check_every, prm->tol * prm->tol, replace2, sign,
               force_global ? 0 : 1, (prm->flags & GF_FLAG_SGS_MASK) >> GF_FLAG_SGS_SHIFT,
               (refined && (prm->flags & GF_FLAG_WARM_START)) ? 1 : 0, c->f.p, c->tile_list,
               c->ny, c->nz, c->nty, c->ntz};
    // the cube-region coarse correction (tile SGS only): set up for the
    // global-memory solve, which runs when forced or when the shared-memory
    // solver defers (the set-up then waits for the same flag)
    if ((prm->flags & GF_FLAG_COARSE) && pa.sgs > 0) {
      const RegionBufs rb = region_bufs(c);
      pa.coarse = 1;
      pa.rg_count = rb.count;
      pa.rg_tiles = rb.tiles;
      pa.rg_of_slot = rb.of_slot;
      pa.rg_nt3 = c->rg.ct * c->rg.ct * c->rg.ct;
      pa.rg_gt = c->rg_gt;
      pa.rg_e = c->rg_e;
      pa.cbuf = c->coarse_buf;
      if ((e = coarse_setup_regions(c, c->state, force_global ? nullptr : &c->state->fallback)))
        return e;
    }
    if (refined) {
      e = launch_pcg<double, true>(c, pa);
      result64 = c->x64;
    } else {
      e = launch_pcg<float, false>(c, pa);
    }
    if (e) return e;
  }
  if (c->timing) cudaEventRecord(c->ev[9], st);
  if ((e = check_cuda(c, cudaMemsetAsync(c->f.p, 0, c->ncell * 4, st), "zero p"))) return e;
  const bool pcg = solver == GF_PCG || solver == GF_PCG_REFINED;
  ScatterArgs sc{c->n_active, c->tile_list, c->code, result, result64, c->f.p,
                 c->ny, c->nz, c->nty, c->ntz, pcg ? c->state : nullptr,
                 pcg ? c->state : nullptr, 1, c->health, c->ncell};
  k_scatter_p<<<gs, 256, 0, st>>>(sc);
  c->launches++;
  c->last_solver = solver;
  return check_launch(c, "gf_pressure");
}

GF_BOUNDS_READER(pressure)

}  // namespace gf
