// Shared-memory-resident preconditioned CG for the pressure system of
// _pressure_pcg (src/gpufluid/solvers/solver3d.py:2917-3043): the same
// operator (diag = #non-solid neighbours, -1 per fluid neighbour), the same
// preconditioner by default (Jacobi, z = r / max(diag, 1); optionally
// tile-local symmetric Gauss-Seidel sweeps) and the same stop test (||r||^2 <
// tol^2 ||r0||^2, checked every check_every iterations), written in the
// single-reduction form of Chronopoulos & Gear (1989): with w = A z,
//   d = z + beta d,  s = w + beta s,  x += alpha d,  r -= alpha s,  z = M r,
//   w = A z,  gamma = r.z,  delta = w.z,
//   beta' = gamma'/gamma,  alpha' = gamma' / (delta' - beta' gamma' / alpha),
// which is algebraically the reference's iteration but needs ONE grid-wide
// reduction per iteration instead of two.
//
// One cooperative block of 1024 threads per SM.  Block b owns the contiguous
// run of active tile slots [b0, b1) (balanced split of n_active) and keeps its
// cells' x, r, d, s, w, stencil codes and a padded 10x10x10 box of z per tile
// in shared memory for the whole solve (plus the FP64 iterate x64 when
// refining).  A tile face whose neighbouring tile belongs to another block is
// a halo face: its fluid cells publish z as tagged 64-bit words (the value's
// bits under a publication count) and the neighbouring block loads them until
// the count matches.  Each iteration: own update -> z = M r -> halo
// publication and ring fill of the z boxes (from the neighbouring tile's box
// or the tagged halo) -> w = A z as a branch-free fixed-offset stencil -> one
// grid all-reduce of (r.z, w.z, r.r).
//
// The grid all-reduce: thread 0 publishes the block's partial sums, arrives
// with a release-ordered add on a monotonic counter and polls it with acquire
// loads (bounded spin); every block then sums all partials in one fixed
// order, so the scalars -- and every decision taken from them -- are the same
// in all blocks and bit-reproducible from run to run.
//
// Refined mode: x accumulates in float32 between FP64 residual replacements
// (x64 += x; r = b - A x64 in FP64) taken whenever ||r|| fell 100x since the
// last one or the float32 recursion claims convergence; the solve ends when
// the FP64 residual meets the target.
//
// If the active region holds more than SmemCfg::MAXT tiles per block the
// kernel sets PcgState::fallback and returns; the global-memory solver (k_pcg
// in pressure.cu) launched right after it then performs the solve.
#include "gf_internal.cuh"

namespace gf {

constexpr int SM_THREADS = 1024;
constexpr long long SM_SPIN_LIMIT = 1LL << 26;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

constexpr int SM_MAXG = 160;      // blocks (one per SM)
constexpr int CRMAX = COARSE_RMAX;  // coarse regions (one per active tile), at most
static_assert(SM_MAXG == COARSE_MAXG, "coarse buffer sizing");

struct GridSync {
  double *partials;            // [2][4][G]
  unsigned long long *counter; // monotonic arrival counter (zeroed per solve)
  int *err;
  unsigned long long epoch;
  long long *trace;            // nullable: SM clock stamps of block 0
  int trace_n, trace_cap;
  long long busy, t_last;      // per-block cycles spent outside the all-reduce
};

__device__ __forceinline__ void trace_mark(GridSync &gs) {
  if (gs.trace && blockIdx.x == 0 && threadIdx.x == 0 && gs.trace_n < gs.trace_cap)
    gs.trace[gs.trace_n++] = clock64();
}

__device__ __forceinline__ void red_release_add(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid-wide sum of NV values; every block obtains the same totals.  Two
// block-level barriers: (1) every warp's shuffle-reduced values land in shared
// memory; then warp 0 alone sums the block's warps, lane 0 publishes the
// block's partials and arrives with a release-ordered add on the monotonic
// counter (after the barrier, so the whole block's earlier global writes are
// ordered before it) and polls it with acquire loads (bounded spin), and warp
// 0 sums all blocks' partials in one fixed order; (2) the totals are
// broadcast.  Every block therefore derives identical scalars, and the
// result is bit-reproducible from run to run.  sh holds >= 36 * NV values.
template <typename T, int NV>
__device__ __forceinline__ bool grid_allreduce(GridSync &gs, const T (&v)[NV], T (&tot)[NV],
                                               T *sh) {
  trace_mark(gs);
  if (gs.trace && threadIdx.x == 0) gs.busy += clock64() - gs.t_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T *s_tot = sh + 32 * NV;  // NV values, alternated by epoch parity below
  const int buf = (int)(gs.epoch & 1ull);
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    T w = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (lane == 0) sh[k * 32 + wid] = w;
  }
  __syncthreads();
  if (wid == 0) {
    const unsigned G = gridDim.x;
    T bsum[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      T t = lane < (int)(blockDim.x >> 5) ? sh[k * 32 + lane] : (T)0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      bsum[k] = t;
    }
    int ok = 1;
    if (lane == 0) {
#pragma unroll
      for (int k = 0; k < NV; ++k) gs.partials[(buf * 4 + k) * G + blockIdx.x] = (double)bsum[k];
      red_release_add(gs.counter, 1ull);
      const unsigned long long target = (gs.epoch + 1ull) * G;
      long long spins = 0;
      while (ld_acquire_u64(gs.counter) < target) {
        if (++spins > SM_SPIN_LIMIT) {
          atomicExch(gs.err, 1);
          ok = 0;
          break;
        }
      }
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok) {
      // fence so that lanes 1..31 read the partials after lane 0's acquire
      __syncwarp();
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double pv[SM_MAXG / 32];
#pragma unroll
        for (int m = 0; m < SM_MAXG / 32; ++m) {
          const unsigned j = lane + 32 * m;
          pv[m] = j < G ? __ldcg(gs.partials + (buf * 4 + k) * G + j) : 0.0;
        }
        T acc = 0;
#pragma unroll
        for (int m = 0; m < SM_MAXG / 32; ++m) acc += (T)pv[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) s_tot[buf * NV + k] = acc;
      }
    }
  }
  gs.epoch++;
  __syncthreads();
  if (*reinterpret_cast<volatile int *>(gs.err)) return false;
#pragma unroll
  for (int k = 0; k < NV; ++k) tot[k] = s_tot[buf * NV + k];
  trace_mark(gs);
  if (gs.trace && threadIdx.x == 0) gs.t_last = clock64();
  return true;
}

// Where the value of neighbour `dir` of local cell L lives: shared memory
// (returns true, Lnb) or another block's halo (returns false, qnb).
__device__ __forceinline__ bool nb_where(int L, int dir, int b0, int b1, const int *s_nbr,
                                         int &Lnb, int64_t &qnb) {
  const int tl = L >> 9, l = L & 511;
  const int li = l >> 6, lj = (l >> 3) & 7, lk = l & 7;
  int off, lw;
  bool inside;
  switch (dir) {
    case 0: inside = li > 0; off = -64; lw = 448 | (l & 63); break;
    case 1: inside = li < 7; off = 64; lw = l & 63; break;
    case 2: inside = lj > 0; off = -8; lw = (l & 0x1C7) | 56; break;
    case 3: inside = lj < 7; off = 8; lw = l & 0x1C7; break;
    case 4: inside = lk > 0; off = -1; lw = l | 7; break;
    default: inside = lk < 7; off = 1; lw = l & ~7; break;
  }
  if (inside) {
    Lnb = L + off;
    return true;
  }
  const int s = s_nbr[tl * 6 + dir];
  if (s >= b0 && s < b1) {
    Lnb = (s - b0) * 512 + lw;
    return true;
  }
  qnb = (int64_t)s * 512 + lw;
  return false;
}

__device__ __forceinline__ bool is_halo(int L, const uint8_t *s_mask) {
  const int l = L & 511, m = s_mask[L >> 9];
  const int li = l >> 6, lj = (l >> 3) & 7, lk = l & 7;
  return (li == 0 && (m & 1)) || (li == 7 && (m & 2)) || (lj == 0 && (m & 4)) ||
         (lj == 7 && (m & 8)) || (lk == 0 && (m & 16)) || (lk == 7 && (m & 32));
}

// Padded-box offsets: a tile's d values live in a 10x10x10 box whose interior
// (1..8)^3 is the tile and whose one-cell ring holds the neighbours' values.
__device__ __forceinline__ int pad_of(int l) {
  return ((l >> 6) + 1) * 100 + (((l >> 3) & 7) + 1) * 10 + ((l & 7) + 1);
}
// Ring position (in the box) and neighbour-tile cell index of face position p
// (0..63) of face `dir`.
__device__ __forceinline__ void face_map(int dir, int p, int &ring, int &lw) {
  const int hi = p >> 3, lo = p & 7;
  switch (dir) {
    case 0: ring = (hi + 1) * 10 + (lo + 1); lw = 448 + p; break;
    case 1: ring = 900 + (hi + 1) * 10 + (lo + 1); lw = p; break;
    case 2: ring = (hi + 1) * 100 + (lo + 1); lw = hi * 64 + 56 + lo; break;
    case 3: ring = (hi + 1) * 100 + 90 + (lo + 1); lw = hi * 64 + lo; break;
    case 4: ring = (hi + 1) * 100 + (lo + 1) * 10; lw = hi * 64 + lo * 8 + 7; break;
    default: ring = (hi + 1) * 100 + (lo + 1) * 10 + 9; lw = hi * 64 + lo * 8; break;
  }
}

// Ring geometry per face direction: ring position base + (hi+1) a + (lo+1) b
// of face position p = hi * 8 + lo, and the offset of the source cell in the
// neighbouring tile's box.
__constant__ int c_ring_base[6] = {0, 900, 0, 90, 0, 9};
__constant__ int c_ring_a[6] = {10, 10, 100, 100, 100, 100};
__constant__ int c_ring_b[6] = {1, 1, 1, 1, 10, 10};
__constant__ int c_ring_delta[6] = {800, -800, 80, -80, 8, -8};

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Face-wise ring fill from tagged halo words (value bits | publication count
// << 32): warp w handles faces f = w, w+32, ... of the block's tiles (f = tile
// * 6 + dir), each lane positions p = lane and lane + 32 of the face, so the
// face's direction and neighbour kind are uniform in the warp.  In-block
// faces are copied box to box; another block's face is loaded
// (both of a lane's words in flight) until both carry the count `ep`.  A
// wait longer than the spin limit sets *err (the next grid reduction then
// ends the solve).
__device__ __forceinline__ void ring_fill_tagged(float *s_zb, const int *s_nbr,
                                                 const int *s_forder, int nface, int b0, int b1,
                                                 const uint8_t *s_rdiag,
                                                 const unsigned long long *hz,
                                                 unsigned long long ep, int *err) {
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = wid; i < nface; i += SM_THREADS / 32) {
    const int f = s_forder[i];
    const int sl = s_nbr[f];
    const int tl = f / 6, dir = f - tl * 6;
    const int base = c_ring_base[dir], ca = c_ring_a[dir], cb = c_ring_b[dir];
    float *dst = s_zb + tl * 1000;
    int ring[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = lane + 32 * h;
      ring[h] = base + ((p >> 3) + 1) * ca + ((p & 7) + 1) * cb;
    }
    if (sl >= b0 && sl < b1) {
      const float *src = s_zb + (sl - b0) * 1000 + c_ring_delta[dir];
      dst[ring[0]] = src[ring[0]];
      dst[ring[1]] = src[ring[1]];
      continue;
    }
    int64_t q[2];
    bool need[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = lane + 32 * h, hi = p >> 3, lo = p & 7;
      int lw;
      switch (dir) {
        case 0: lw = 448 + p; break;
        case 1: lw = p; break;
        case 2: lw = hi * 64 + 56 + lo; break;
        case 3: lw = hi * 64 + lo; break;
        case 4: lw = hi * 64 + lo * 8 + 7; break;
        default: lw = hi * 64 + lo * 8; break;
      }
      q[h] = (int64_t)sl * 512 + lw;
      need[h] = s_rdiag[f * 64 + p] != 0;  // non-fluid remote cells read as 0
    }
    unsigned long long w0 = need[0] ? ld_relaxed_u64(hz + q[0]) : 0ull;
    unsigned long long w1 = need[1] ? ld_relaxed_u64(hz + q[1]) : 0ull;
    long long spins = 0;
    while ((need[0] && (w0 >> 32) != ep) || (need[1] && (w1 >> 32) != ep)) {
      if (++spins > SM_SPIN_LIMIT) {
        atomicExch(err, 1);
        break;
      }
      if (need[0] && (w0 >> 32) != ep) w0 = ld_relaxed_u64(hz + q[0]);
      if (need[1] && (w1 >> 32) != ep) w1 = ld_relaxed_u64(hz + q[1]);
    }
    dst[ring[0]] = need[0] ? __uint_as_float((unsigned)w0) : 0.f;
    dst[ring[1]] = need[1] ? __uint_as_float((unsigned)w1) : 0.f;
  }
}

// One-round-trip grid sum of the three scalars of an iteration.  No halo
// data rides on it (the halo words carry their own counts), so it needs no
// fence: warp 0 publishes the block's three sums as float32 payloads under a
// 32-bit epoch count in three 64-bit words (relaxed stores, double-buffered by
// epoch parity), and lane t of warps 0-1 reads the words of blocks t, t+64,
// t+128 -- all in flight -- until every count matches (bounded spin).  Each
// lane adds its blocks in order, the warps shuffle-reduce, and the two warps'
// sums are added in warp order, so every block derives the same totals.  The
// per-block sums travel as float32 (relative rounding 6e-8); the refined
// solve's accuracy rests on its FP64 residual replacements, not on these.
constexpr int FAST_WORDS = 4;  // words per block and parity (3 used)
constexpr int64_t FAST_SLOTS_OFF = 2048;  // in doubles, into the partials buffer
// tagged coarse sums g_t: [2][CRMAX] u64 after the reduction words
constexpr int64_t COARSE_SLOTS_OFF = FAST_SLOTS_OFF + 2 * 160 * FAST_WORDS;
static_assert(COARSE_SLOTS_OFF + 2 * CRMAX <= 3 * MAX_PCG_BLOCKS, "partials buffer");
struct FastSync {
  unsigned long long *slots;  // [2][SM_MAXG][FAST_WORDS], zeroed per solve
  unsigned long long epoch;
  int *err;
  long long spin_limit;       // polls before a wait gives up
  int stall;                  // test only: the first reduction waits for a count nobody publishes
};

template <typename T>
__device__ __forceinline__ bool fast_allreduce3(FastSync &fs, GridSync &gs, const T (&v)[3],
                                                T (&tot)[3], T *sh) {
  trace_mark(gs);
  if (gs.trace && threadIdx.x == 0) gs.busy += clock64() - gs.t_last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T *s_two = sh + 96;  // [2][3] per-warp totals
  const unsigned G = gridDim.x;
  const unsigned long long tag = ((fs.epoch + 1ull) & 0xffffffffull) << 32;
  // the count the readers wait for; under the test stall the first reduction
  // waits for the next epoch's count, which no block publishes before every
  // block has left this one, so every wait runs out
  const unsigned long long want = (fs.stall && fs.epoch == 0ull) ? tag + (1ull << 32) : tag;
  unsigned long long *slots = fs.slots + (fs.epoch & 1ull) * (SM_MAXG * FAST_WORDS);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T w = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if (lane == 0) sh[k * 32 + wid] = w;
  }
  __syncthreads();
  if (wid == 0) {
    T t0 = sh[lane], t1 = sh[32 + lane], t2 = sh[64 + lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      t0 += __shfl_down_sync(0xffffffffu, t0, o);
      t1 += __shfl_down_sync(0xffffffffu, t1, o);
      t2 += __shfl_down_sync(0xffffffffu, t2, o);
    }
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    t1 = __shfl_sync(0xffffffffu, t1, 0);
    t2 = __shfl_sync(0xffffffffu, t2, 0);
    if (lane < 3) {
      const float f = (float)(lane == 0 ? t0 : (lane == 1 ? t1 : t2));
      st_relaxed_u64(slots + blockIdx.x * FAST_WORDS + lane, tag | __float_as_uint(f));
    }
  }
  if (wid < 2) {
    const unsigned idx = threadIdx.x;
    bool need[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) need[m] = idx + 64u * m < G;
    unsigned long long w[3][3];
    long long spins = 0;
    for (;;) {
      bool all = true;
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          w[m][k] = need[m] ? ld_relaxed_u64(slots + (idx + 64u * m) * FAST_WORDS + k) : want;
          all &= (w[m][k] & 0xffffffff00000000ull) == want;
        }
      if (all) break;
      if (++spins > fs.spin_limit) {
        atomicExch(fs.err, 1);
        break;
      }
    }
    T acc[3] = {(T)0, (T)0, (T)0};
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (need[m]) acc[k] += (T)__uint_as_float((unsigned)w[m][k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T t = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) s_two[wid * 3 + k] = t;
    }
  }
  fs.epoch++;
  __syncthreads();
  if (*reinterpret_cast<volatile int *>(fs.err)) return false;
#pragma unroll
  for (int k = 0; k < 3; ++k) tot[k] = s_two[k] + s_two[3 + k];
  trace_mark(gs);
  if (gs.trace && threadIdx.x == 0) gs.t_last = clock64();
  return true;
}

template <bool REF>
struct SmemCfg {
  // per tile: x, r, d, s, w (2048 B each), padded z box (4000 B), code
  // (1024 B), remote ring diagonals (384 B), x64 (4096 B, refined).  Shared
  // memory holds all per-cell state so that no register array spills: with
  // ~227 KB of the SM's on-chip memory in use, L1 is too small to absorb spills.
  static constexpr size_t TILE_BYTES = 5 * 2048 + 4000 + 1024 + 384 + (REF ? 4096 : 0);
  static constexpr int MAXT = REF ? 11 : 14;  // tiles per block (<= 227 KB with statics)
  static constexpr int MAXJ = (MAXT * 512 + SM_THREADS - 1) / SM_THREADS;
  static constexpr size_t BYTES = (size_t)MAXT * TILE_BYTES;
};

__device__ __forceinline__ float diagz_of(uint16_t code) {
  return fmaxf((float)((code >> CODE_DIAG_SHIFT) & 7), 1.0f);
}

// Block boundaries over the active slots, balanced by the per-slot work
// estimate (fluid cells + ring) and identical in every block; falls back to
// an equal split of slots when the balanced split would give some block more
// than maxt tiles.  Uses `scratch` (>= na ints of shared memory).
__device__ void partition_slots(const int32_t *__restrict__ cost, int na, int maxt, int *scratch,
                                int *s_bounds) {
  const int G = gridDim.x;
  // inclusive prefix of the costs (chunked block scan)
  __shared__ int carry, warp_sums[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int off = 0; off < na; off += blockDim.x) {
    const int t = off + threadIdx.x;
    const int v = t < na ? cost[t] : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int sv = lane < nw ? warp_sums[lane] : 0;
      int si = sv;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += u;
      }
      if (lane < nw) warp_sums[lane] = si - sv;
    }
    __syncthreads();
    if (t < na) scratch[t] = carry + warp_sums[wid] + incl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += warp_sums[wid] + incl;
    __syncthreads();
  }
  const long long total = na > 0 ? scratch[na - 1] : 0;
  // bound[g] = first slot whose inclusive prefix exceeds total * g / G
  for (int g = threadIdx.x; g <= G; g += blockDim.x) {
    int lo = 0, hi = na;
    const long long target = total * g / G;
    if (g == G) {
      lo = na;
    } else {
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((long long)scratch[mid] <= target) lo = mid + 1; else hi = mid;
      }
      if (g == 0) lo = 0;
    }
    s_bounds[g] = lo;
  }
  __syncthreads();
  int ok = 1;
  for (int g = threadIdx.x; g < G; g += blockDim.x)
    if (s_bounds[g + 1] - s_bounds[g] > maxt || s_bounds[g + 1] < s_bounds[g]) ok = 0;
  ok = __syncthreads_and(ok);
  if (!ok)
    for (int g = threadIdx.x; g <= G; g += blockDim.x) s_bounds[g] = (int)((long long)g * na / G);
  __syncthreads();
}

template <typename Acc, bool REF, bool SGS, bool CRS>
__global__ void __launch_bounds__(SM_THREADS, 1) k_pcg_smem(PcgSmemArgs a) {
  using Cfg = SmemCfg<REF>;
  constexpr int MAXT = Cfg::MAXT, MAXJ = Cfg::MAXJ;
  static_assert(MAXJ * 3 <= 32, "diagonal pack");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int s_nbr[MAXT * 6];
  __shared__ float s_rtab[16];  // by (fluid << 3 | count): 0, or 1 / max(count, 1)
  __shared__ uint8_t s_mask[MAXT];
  __shared__ int s_forder[MAXT * 6];  // faces with a neighbouring tile, another block's first
  __shared__ int s_nface;
  __shared__ int s_bounds[SM_MAXG + 1];
  __shared__ Acc sh[36 * 4];
  __shared__ double shd[36 * 4];
  // coarse correction: warp partials of e_t = B_t . g, and of the tiles'
  // residual sums g_t (16 warps per tile)
  __shared__ float s_ep[32];
  __shared__ float s_gw[MAXT * 16];

  PcgState *st = a.st;
  const int na = *a.n_active;
  const int G = gridDim.x;
  if (na > G * MAXT) {  // does not fit: the global-memory solver takes over
    if (blockIdx.x == 0 && threadIdx.x == 0) st->fallback = 1;
    return;
  }
  GridSync gs{a.partials, a.counter, &st->error, 0ull, a.trace, 0, a.trace_cap / 2, 0, clock64()};
  FastSync fs{reinterpret_cast<unsigned long long *>(a.partials + FAST_SLOTS_OFF), 0ull,
              &st->error, a.test_stall ? 4096ll : SM_SPIN_LIMIT, a.test_stall};
  // Phases of an iteration for the trace (block thread 0's view, cycles):
  // 0 own update, 1 SGS sweeps, 2 halo publication + neighbour flags +
  // in-block rings, 3 remote rings, 4 stencil and dot products, 5 grid
  // all-reduce (with the barrier before it), 6 coarse gather of the tiles'
  // residual sums (the wait for their publication), 7 coarse e = B g and its
  // addition to z.  s_ph[8] holds the last stamp.
  __shared__ long long s_ph[9];
  if (threadIdx.x == 0)
    for (int k = 0; k < 9; ++k) s_ph[k] = k < 8 ? 0 : clock64();
  auto phase_mark = [&](int k) {
    if (a.trace && threadIdx.x == 0) {
      const long long now = clock64();
      s_ph[k] += now - s_ph[8];
      s_ph[8] = now;
    }
  };
  if (G > SM_MAXG) {
    if (threadIdx.x == 0) atomicExch(&st->error, 1);
    return;
  }
  // the per-cell arrays are not yet in use: borrow their memory for the
  // partition prefix
  partition_slots(a.tile_cost, na, MAXT, reinterpret_cast<int *>(smem), s_bounds);
  const int b0 = s_bounds[blockIdx.x], b1 = s_bounds[blockIdx.x + 1];
  const int nt = b1 - b0;
  const int64_t q0 = (int64_t)b0 * 512;
  // per-cell arrays pitched by this block's tile count, so that the memory of
  // its MAXT - nt unused tiles is one free region at the end (16-byte aligned:
  // every array's size per tile is a multiple of 16 bytes)
  unsigned char *pb = smem;
  double *s_x64 = reinterpret_cast<double *>(pb);
  if (REF) pb += (size_t)nt * 4096;
  float *s_x = reinterpret_cast<float *>(pb);
  float *s_r = s_x + nt * 512;
  float *s_d = s_r + nt * 512;
  float *s_s = s_d + nt * 512;
  float *s_w = s_s + nt * 512;
  // w doubles as the gathered coarse residual sums (one per active tile,
  // rounded up to 8), so it spans at least that many floats; the layout still
  // fits, since a block holding fewer than MAXT tiles has a whole free tile
  // (over 19 KB) and the sums take at most 160 * 14 floats (8.75 KB)
  const int wlen = nt * 512 > ((na + 7) & ~7) ? nt * 512 : ((na + 7) & ~7);
  float *s_zb = s_w + wlen;  // padded z boxes, 1000 per tile
  uint16_t *s_code = reinterpret_cast<uint16_t *>(s_zb + nt * 1000);
  uint8_t *s_rdiag = reinterpret_cast<uint8_t *>(s_code + nt * 512);  // 384 per tile
  unsigned char *const s_free = s_rdiag + nt * 384;
  const size_t used = (size_t)(s_free - smem);
  const size_t free_bytes = used < Cfg::BYTES ? Cfg::BYTES - used : 0;
  static_assert(Cfg::TILE_BYTES % 16 == 0, "free region alignment");

  const int l = threadIdx.x & 511, tl0 = threadIdx.x >> 9;
  const int pc = pad_of(l);

  // ---- coarse correction (GF_FLAG_COARSE): one region per active tile, P
  // the indicator of each tile's fluid cells, and the preconditioner
  // M^-1 = M_tile^-1 + P B P^T (additive two-level) with B = (P^T A P)^-1,
  // whose rows the set-up kernels of coarse.cu computed before this launch (as
  // bfloat16; the set CoarseMeta::parity names).  A failed row solve switched
  // the correction off for the solve.
  const bool coarse = CRS && a.coarse && a.cbuf != nullptr &&
                      *reinterpret_cast<volatile int *>(&st->coarse_off) == 0;
  const uint16_t *const Bh =
      coarse ? reinterpret_cast<const uint16_t *>(a.cbuf) +
                   (int64_t)reinterpret_cast<const CoarseMeta *>(a.cbuf + COARSE_META_OFF)->parity *
                       CRMAX * CRMAX
             : nullptr;
  // this block's rows of B (R8 bf16 each), copied once into the free region
  // when they fit, so that e = B g reads shared memory instead of L2
  const int R8c = (na + 7) & ~7;
  const bool b_smem = coarse && (size_t)nt * R8c * 2 <= free_bytes;
  uint4 *const s_B = reinterpret_cast<uint4 *>(s_free);
  if (b_smem) {
    const int nch = R8c >> 3;
    for (int i = threadIdx.x; i < nt * nch; i += blockDim.x) {
      const int jr = i / nch, ch = i - jr * nch;
      s_B[i] = __ldg(reinterpret_cast<const uint4 *>(Bh + (int64_t)(b0 + jr) * CRMAX) + ch);
    }
  }

  for (int i = threadIdx.x; i < nt * 6; i += blockDim.x) s_nbr[i] = a.nbr[(int64_t)b0 * 6 + i];
  for (int i = threadIdx.x; i < nt * 1000; i += blockDim.x) s_zb[i] = 0.f;
  if (threadIdx.x < 16)
    s_rtab[threadIdx.x] = threadIdx.x < 8 ? 0.f : 1.0f / fmaxf((float)(threadIdx.x - 8), 1.0f);
  __syncthreads();
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    int m = 0;
    for (int dir = 0; dir < 6; ++dir) {
      const int sl = s_nbr[t * 6 + dir];
      if (sl >= 0 && (sl < b0 || sl >= b1)) m |= 1 << dir;
    }
    s_mask[t] = (uint8_t)m;
  }
  if (threadIdx.x == 0) {  // remote faces lead, so each warp starts with at most one
    int n = 0;
    for (int pass = 0; pass < 2; ++pass)
      for (int f = 0; f < nt * 6; ++f) {
        const int sl = s_nbr[f];
        if (sl < 0) continue;
        const bool remote = sl < b0 || sl >= b1;
        if (remote == (pass == 0)) s_forder[n++] = f;
      }
    s_nface = n;
  }
  // diagonal (max(count,1)) of remote ring cells, 0 when not fluid
  for (int w = threadIdx.x; w < nt * 384; w += SM_THREADS) {
    const int tl = w / 384, rem = w - tl * 384, dir = rem >> 6, p = rem & 63;
    int ring, lw;
    face_map(dir, p, ring, lw);
    const int sl = s_nbr[tl * 6 + dir];
    uint8_t dg = 0;
    if (sl >= 0 && (sl < b0 || sl >= b1)) {
      const uint16_t cd = a.code[(int64_t)sl * 512 + lw];
      if (cd & CODE_FLUID) dg = (uint8_t)diagz_of(cd);
    }
    s_rdiag[w] = dg;
  }
  __syncthreads();
  // sweeps of the tile SGS preconditioner; 0: Jacobi (the reference's), for
  // which the instantiation carries no sweep code
  const int sgs = SGS ? a.sgs_sweeps : 0;

  // ---- init: r0 = b, z0 = M r0, w0 = A z0; d_{-1} = s_{-1} = 0.  Per-thread
  // masks: fluid (bit j), halo (bit j), neighbour count (3 bits per j).
  unsigned fmask = 0, hmask = 0, dpack = 0;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // warp partial of the tile's residual sum g_t (a barrier follows before use)
  auto tile_partial = [&](int tl, float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) s_gw[tl * 16 + (wid & 15)] = v;
  };

  // the warp partials of all the thread's tiles at once (v[j] for tile tl0 +
  // 2j, 0 beyond the block's tiles): a butterfly over eight values -- three
  // exchange levels that halve the values a lane holds, then two plain levels
  // -- leaves lane L with the warp's sum of value (L >> 2) & 7 after 9
  // shuffles instead of 5 per tile; lane 4q writes value q
  auto tile_partials = [&](const float (&v)[MAXJ]) {
    static_assert(MAXJ <= 8, "eight values per butterfly");
    float a8[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a8[q] = q < MAXJ ? v[q < MAXJ ? q : 0] : 0.f;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    float w4[4], w2[2];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      w4[q] = (b4 ? a8[4 + q] : a8[q]) +
              __shfl_xor_sync(0xffffffffu, b4 ? a8[q] : a8[4 + q], 16);
#pragma unroll
    for (int q = 0; q < 2; ++q)
      w2[q] = (b3 ? w4[2 + q] : w4[q]) +
              __shfl_xor_sync(0xffffffffu, b3 ? w4[q] : w4[2 + q], 8);
    float y = (b2 ? w2[1] : w2[0]) + __shfl_xor_sync(0xffffffffu, b2 ? w2[0] : w2[1], 4);
    y += __shfl_xor_sync(0xffffffffu, y, 2);
    y += __shfl_xor_sync(0xffffffffu, y, 1);
    const int q = (lane >> 2) & 7, tl = tl0 + 2 * q;
    if ((lane & 3) == 0 && q < MAXJ && tl < nt) s_gw[tl * 16 + (wid & 15)] = y;
  };
  // warm start (refined only): x64 = the dense p0 at the cell, r = b - A x64
  // in FP64 with the neighbours' p0 read from the dense array (complete and
  // read-only during the solve, so no halo exchange); the stop test stays
  // relative to ||b||, so the accuracy target is the cold start's
  const bool warm = REF && a.warm && a.p0 != nullptr;
  double wb2 = 0.0, wr2 = 0.0;  // this thread's sums of b^2 and r0^2
#pragma unroll
  for (int j = 0; j < MAXJ; ++j) {
    const int tl = tl0 + 2 * j;
    if (tl >= nt) break;
    const int L = tl * 512 + l;
    const uint16_t code = a.code[q0 + L];
    s_code[L] = code;
    float b = 0.f;
    double x0 = 0.0;
    if (code & CODE_FLUID) {
      fmask |= 1u << j;
      dpack |= (unsigned)((code >> CODE_DIAG_SHIFT) & 7) << (3 * j);
      b = a.sign * a.bdiv[q0 + L];
      if (warm) {
        const int t = a.tile_list[b0 + tl];
        const int ti = t / (a.nty * a.ntz), tj = (t / a.ntz) % a.nty, tk = t % a.ntz;
        const int64_t sI = (int64_t)a.ny * a.nz;
        const int64_t g = (int64_t)(ti * 8 + (l >> 6)) * sI + (tj * 8 + ((l >> 3) & 7)) * a.nz +
                          (tk * 8 + (l & 7));
        x0 = (double)a.p0[g];
        const int64_t off[6] = {-sI, sI, -(int64_t)a.nz, (int64_t)a.nz, -1, 1};
        double sum = 0.0;
#pragma unroll
        for (int dir = 0; dir < 6; ++dir)
          if (code & (1 << dir)) sum += (double)a.p0[g + off[dir]];
        const double res = (double)b - ((double)((code >> CODE_DIAG_SHIFT) & 7) * x0 - sum);
        wb2 += (double)b * (double)b;
        wr2 += res * res;
        b = (float)res;  // from here on, the initial residual
      }
      s_zb[tl * 1000 + pc] =
          SGS ? b * s_rtab[8 | ((code >> CODE_DIAG_SHIFT) & 7)] : b / diagz_of(code);
      if (is_halo(L, s_mask)) hmask |= 1u << j;
    }
    s_r[L] = b;
    s_x[L] = 0.f;
    s_d[L] = 0.f;
    s_s[L] = 0.f;
    if (REF) s_x64[L] = x0;
    if (CRS && coarse) tile_partial(tl, b);
  }
  __syncthreads();

  // ---- z = M r and its ring.  Jacobi (sgs == 0): z = r/D, written by the
  // callers.  Tile-local symmetric Gauss-Seidel (sgs sweeps): z = M r with
  // M^-1 = sweeps of red-black symmetric Gauss-Seidel on each 8^3 tile from
  // z = 0, the tile's neighbours held at 0 (the diagonal block of A per tile;
  // symmetric positive definite, so CG applies).  The first red half-sweep
  // (z = r/D) is the z = r/D every caller writes for all fluid cells; then
  // per sweep black, red.  Callers also zero the boxes' rings, and non-fluid
  // cells hold 0, so a half-sweep is the branch-free six-neighbour sum with a
  // per-cell factor (0 on non-fluid cells).  It maps thread t to cell
  // sgs_color_cell(t & 255) of the colour (bank-conflict-free in the boxes)
  // in tiles (t >> 8) + 4i, so all threads work.  The result is published on
  // the halo cells as 64-bit words, the
  // float's bits under a 32-bit publication count (relaxed stores: the word
  // is its own flag, no fence), and the ring of another block's tile is
  // loaded until the count matches (bounded).  The words are zeroed before
  // every solve.  A word is overwritten only after the reduction that
  // follows its reads, so no publication is missed.
  unsigned long long zep = 0;  // z publications, the same sequence in every block
  unsigned long long *const HZ = reinterpret_cast<unsigned long long *>(a.hr0);
  auto half_sweep = [&](int c) {  // z = (r + in-tile fluid neighbours' z) / D, colour c
    const int lc = sgs_color_cell(threadIdx.x & 255, c);
    const int pcc = pad_of(lc);
    for (int tl = threadIdx.x >> 8; tl < nt; tl += 4) {
      const int L = tl * 512 + lc;
      const unsigned code = s_code[L];
      float *zp = s_zb + tl * 1000 + pcc;
      float acc = s_r[L];
      acc = acc + zp[-100];
      acc = acc + zp[100];
      acc = acc + zp[-10];
      acc = acc + zp[10];
      acc = acc + zp[-1];
      acc = acc + zp[1];
      *zp = acc * s_rtab[((code >> 12) & 8) | ((code >> CODE_DIAG_SHIFT) & 7)];
    }
  };
  auto zero_rings = [&]() {  // faces with a neighbouring tile (the others stay 0)
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = wid; i < s_nface; i += SM_THREADS / 32) {
      const int f = s_forder[i];
      const int tl = f / 6, dir = f - tl * 6;
      const int base = c_ring_base[dir], ca = c_ring_a[dir], cb = c_ring_b[dir];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int p = lane + 32 * h;
        s_zb[tl * 1000 + base + ((p >> 3) + 1) * ca + ((p & 7) + 1) * cb] = 0.f;
      }
    }
  };
  // Callers have written z = r/D on their fluid cells, zeroed the rings
  // (zero_rings, SGS only) and passed a barrier.
  // Coarse correction: each block publishes its tiles' residual sums g_t as
  // tagged words before the sweeps and gathers all of them (inside the last
  // sweep with two or more sweeps, else after the sweeps) into the w array,
  // which is free until the stencil rebuilds it; then e_t = B_t . g for its
  // tiles (bf16 rows of B from shared memory or L2, several warps per row, a
  // fixed-order sum) is added to the z of each tile's fluid cells after the
  // sweeps, so the halo exchange, the stencil and the dot products below all
  // see u = z + P e.
  unsigned long long gep = 0;  // g publications, the same sequence in every block
  unsigned long long *const GSL =
      reinterpret_cast<unsigned long long *>(a.partials + COARSE_SLOTS_OFF);
  auto precond_exchange = [&]() {
    if (CRS && coarse && (int)threadIdx.x < nt) {  // publish g_t for the block's tiles
      float g = 0.f;
#pragma unroll
      for (int w = 0; w < 16; ++w) g += s_gw[threadIdx.x * 16 + w];
      st_relaxed_u64(GSL + (gep & 1ull) * CRMAX + b0 + threadIdx.x,
                     ((gep + 1ull) << 32) | __float_as_uint(g));
    }
    // thread t gathers the words of tiles t, t + 1024, t + 2048; the first
    // loads are issued a half-sweep before the words are needed, so their
    // latency hides behind it; a stale word is polled again
    const unsigned long long *gsrc = GSL + (gep & 1ull) * CRMAX;
    const int t = threadIdx.x;
    unsigned long long gpre[3] = {0ull, 0ull, 0ull};
    auto prefetch = [&]() {
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (t + k * SM_THREADS < na) gpre[k] = ld_relaxed_u64(gsrc + t + k * SM_THREADS);
    };
    const unsigned long long gtag = (gep + 1ull) << 32;
    float *const s_g = s_w;  // [R8]: the gathered g, zero-padded
    const int R8 = (na + 7) & ~7;
    // wait for every tile's g_t word (bounded) and store the sums into s_g
    auto gather_store = [&]() {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const int sl = t + k * SM_THREADS;
        if (sl < na) {
          unsigned long long w = gpre[k];
          long long spins = 0;
          while ((w & 0xffffffff00000000ull) != gtag) {
            w = ld_relaxed_u64(gsrc + sl);
            if ((w & 0xffffffff00000000ull) == gtag) break;
            if (++spins > SM_SPIN_LIMIT) {
              atomicExch(&st->error, 1);
              w = 0;
              break;
            }
          }
          s_g[sl] = __uint_as_float((unsigned)w);
        } else if (sl < R8) {
          s_g[sl] = 0.f;
        }
      }
      ++gep;
    };
    // this warp's share of e_t = B_t . g (s_g complete): row b0 + jr is summed
    // by warps jr, jr + nt, ... (the lanes over 8-column chunks)
    auto e_chunks = [&](float &v) {
      if (nt <= 0) return;
      const int jr = wid % nt, iw = wid / nt, nw = (31 - jr) / nt + 1;
      const uint4 *row = b_smem ? s_B + jr * (R8 >> 3)
                                : reinterpret_cast<const uint4 *>(Bh + (int64_t)(b0 + jr) * CRMAX);
      auto ldB = [&](int ch) -> uint4 { return b_smem ? row[ch] : __ldg(row + ch); };
      auto dot8 = [&](const uint4 q, int ch) {
        const float *gp = s_g + ch * 8;
        v += __uint_as_float(q.x << 16) * gp[0] + __uint_as_float(q.x & 0xffff0000u) * gp[1];
        v += __uint_as_float(q.y << 16) * gp[2] + __uint_as_float(q.y & 0xffff0000u) * gp[3];
        v += __uint_as_float(q.z << 16) * gp[4] + __uint_as_float(q.z & 0xffff0000u) * gp[5];
        v += __uint_as_float(q.w << 16) * gp[6] + __uint_as_float(q.w & 0xffff0000u) * gp[7];
      };
      // two chunks in flight per lane, so a lane's loads wait one L2 trip
      const int nch = R8 >> 3, step = nw * 32;
      int ch = iw * 32 + lane;
      for (; ch + step < nch; ch += 2 * step) {
        const uint4 q0 = ldB(ch), q1 = ldB(ch + step);
        dot8(q0, ch);
        dot8(q1, ch + step);
      }
      if (ch < nch) dot8(ldB(ch), ch);
    };
    // the warp's partial of its row, for the sums in warp order below
    auto e_reduce = [&](float v) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) s_ep[wid] = v;
    };
    // With two or more sweeps the coarse work rides inside the last sweep (it
    // does not depend on the sweeps: M^-1 is the sum of the two parts): the g
    // words are loaded before the last sweep and stored after its first
    // half-sweep, before that barrier (published all earlier half-sweeps ago,
    // so the wait is short); the last half-sweep starts with the e = B g
    // products and ends with their warp sums.  This saves the two block
    // barriers of the gather and of the products and lets their latency
    // overlap the sweeps (measured 17.4 -> 16.9 us per iteration at 128^3).
    const bool early = CRS && coarse && sgs >= 2;
    if (early) {
      for (int sw = 0; sw < sgs - 1; ++sw) {
        half_sweep(1);
        __syncthreads();
        if (sw == sgs - 2) prefetch();
        half_sweep(0);
        __syncthreads();
      }
      half_sweep(1);
      gather_store();
      __syncthreads();
      {
        float ev = 0.f;
        e_chunks(ev);
        half_sweep(0);
        e_reduce(ev);
        __syncthreads();
      }
    } else {
      for (int sw = 0; sw < sgs; ++sw) {
        half_sweep(1);
        __syncthreads();
        if (CRS && coarse && sw == sgs - 1) prefetch();
        half_sweep(0);
        __syncthreads();
      }
    }
    phase_mark(1);
    if (CRS && coarse) {
      if (!early) {
        if (sgs == 0) prefetch();
        gather_store();
        __syncthreads();
        phase_mark(6);
        float ev = 0.f;
        e_chunks(ev);
        e_reduce(ev);
        __syncthreads();
      }
      // lane t < nt of every warp sums e_t from the warps' partials (in warp
      // order); a thread's tiles tl0 + 2j are the same across its warp, so
      // each takes its e_t from lane tl by a shuffle
      float e_lane = 0.f;
      if (lane < nt)
        for (int w = lane; w < 32; w += nt) e_lane += s_ep[w];
#pragma unroll
      for (int j = 0; j < MAXJ; ++j) {
        const int tl = tl0 + 2 * j;
        const float e = __shfl_sync(0xffffffffu, e_lane, tl & 31);
        if ((fmask >> j) & 1) s_zb[tl * 1000 + pc] += e;
      }
      __syncthreads();
    }
    phase_mark(7);
    ++zep;
    const unsigned long long tag = zep << 32;
#pragma unroll
    for (int j = 0; j < MAXJ; ++j)
      if ((hmask >> j) & 1)
        st_relaxed_u64(HZ + q0 + (tl0 + 2 * j) * 512 + l,
                       tag | __float_as_uint(s_zb[(tl0 + 2 * j) * 1000 + pc]));
    phase_mark(2);
    ring_fill_tagged(s_zb, s_nbr, s_forder, s_nface, b0, b1, s_rdiag, HZ, zep, &st->error);
    __syncthreads();
    phase_mark(3);
  };

  precond_exchange();

  // w = A z for own fluid cells (non-fluid box entries are exactly 0, so the
  // branch-free six-neighbour sum equals the reference's fluid-only sum)
  auto stencil = [&](int j, float &z) -> float {
    const float *zp = s_zb + (tl0 + 2 * j) * 1000 + pc;
    float acc = zp[-100];
    acc = acc + zp[100];
    acc = acc + zp[-10];
    acc = acc + zp[10];
    acc = acc + zp[-1];
    acc = acc + zp[1];
    z = *zp;
    return (float)((dpack >> (3 * j)) & 7) * z - acc;
  };
  Acc v3[3] = {0, 0, 0};
#pragma unroll
  for (int j = 0; j < MAXJ; ++j) {
    if (!((fmask >> j) & 1)) continue;
    const int L = (tl0 + 2 * j) * 512 + l;
    float z;
    const float wn = stencil(j, z);
    const float r = s_r[L];
    s_w[L] = wn;
    v3[0] += (Acc)(r * z);
    v3[1] += (Acc)(wn * z);
    v3[2] += (Acc)(r * r);
  }
  Acc t3[3];
  if (!fast_allreduce3<Acc>(fs, gs, v3, t3, sh)) return;
  double wtot[2] = {0.0, 0.0};
  if (warm) {  // ||b||^2 and the FP64 ||b - A x0||^2 of the warm start
    const double wv[2] = {wb2, wr2};
    if (!grid_allreduce<double, 2>(gs, wv, wtot, shd)) return;
  }
  Acc gamma = t3[0];
  const Acc r0 = t3[2];
  const double b2 = warm ? wtot[0] : (double)t3[2];
  double r_upd2 = (double)t3[2], r_true2 = warm ? wtot[1] : b2, rr_last = (double)t3[2];
  Acc alpha = fabs((double)t3[1]) < 1.0e-30 ? (Acc)0 : gamma / t3[1];
  Acc beta = 0;
  int done = warm ? (b2 < 1e-30 || r_true2 <= a.tol2 * b2 ? 1 : 0) : ((double)r0 < 1e-30 ? 1 : 0);
  int iters = 0, nrep = 0, status = GF_OK;

  for (int it = 0; it < a.max_iter && !done; ++it) {
    const float alphaf = (float)alpha, nalpha = -alphaf, betaf = (float)beta;
    // ---- own: d = z + beta d; s = w + beta s; x += alpha d; r -= alpha s; z = M r
    float rv[MAXJ];  // new residuals of the thread's cells (0 off the fluid)
#pragma unroll
    for (int j = 0; j < MAXJ; ++j) {
      const int tl = tl0 + 2 * j, L = tl * 512 + l;
      float rn = 0.f;
      if ((fmask >> j) & 1) {
        float *zp = s_zb + tl * 1000 + pc;
        const float dn = *zp + betaf * s_d[L];
        const float sn = s_w[L] + betaf * s_s[L];
        s_d[L] = dn;
        s_s[L] = sn;
        s_x[L] = s_x[L] + alphaf * dn;
        rn = s_r[L] + nalpha * sn;
        s_r[L] = rn;
        *zp = SGS ? rn * s_rtab[8 | ((dpack >> (3 * j)) & 7)]
                  : rn / fmaxf((float)((dpack >> (3 * j)) & 7), 1.0f);
      }
      rv[j] = rn;
    }
    if (CRS && coarse) tile_partials(rv);
    if (SGS) zero_rings();
    __syncthreads();
    trace_mark(gs);
    phase_mark(0);
    precond_exchange();
    trace_mark(gs);
    // ---- w = A z and the three dot products
    Acc vv[3] = {0, 0, 0};
#pragma unroll
    for (int j = 0; j < MAXJ; ++j) {
      if (!((fmask >> j) & 1)) continue;
      const int L = (tl0 + 2 * j) * 512 + l;
      float z;
      const float wn = stencil(j, z);
      const float r = s_r[L];
      s_w[L] = wn;
      vv[0] += (Acc)(r * z);
      vv[1] += (Acc)(wn * z);
      vv[2] += (Acc)(r * r);
    }
    phase_mark(4);
    Acc tv[3];
    if (!fast_allreduce3<Acc>(fs, gs, vv, tv, sh)) return;
    phase_mark(5);
    iters = it + 1;
    double rr = (double)tv[2];
    rr_last = rr;
    if (!(rr == rr) || !((double)tv[1] == (double)tv[1])) {
      status = GF_NAN;
      done = 1;
      break;
    }
    bool replace = false;
    if (REF) {
      replace = rr < a.replace2 * r_upd2 || rr < a.tol2 * b2;
    } else {
      const bool check = (iters % a.check_every) == 0 || iters == a.max_iter;
      if (check && rr < a.tol2 * (double)r0) done = 1;
    }
    if (REF && replace) {
      // ---- FP64 residual replacement: x64 += x, x = 0; r = b - A x64
#pragma unroll
      for (int j = 0; j < MAXJ; ++j) {
        if (!((fmask >> j) & 1)) continue;
        const int L = (tl0 + 2 * j) * 512 + l;
        const double x64 = s_x64[L] + (double)s_x[L];
        s_x64[L] = x64;
        s_x[L] = 0.f;
        if ((hmask >> j) & 1) a.x64[q0 + L] = x64;
      }
      {
        double z0[1] = {0.0}, zt[1];
        if (!grid_allreduce<double, 1>(gs, z0, zt, shd)) return;
      }
      double vr[1] = {0.0};
#pragma unroll
      for (int j = 0; j < MAXJ; ++j) {
        const int tl = tl0 + 2 * j, L = tl * 512 + l;
        float rf = 0.f;
        if ((fmask >> j) & 1) {
          const uint16_t code = s_code[L];
          double sum = 0.0;
#pragma unroll
          for (int dir = 0; dir < 6; ++dir)
            if (code & (1 << dir)) {
              int Lnb;
              int64_t qnb;
              sum += nb_where(L, dir, b0, b1, s_nbr, Lnb, qnb) ? s_x64[Lnb] : __ldcg(a.x64 + qnb);
            }
          const double diag = (double)((code >> CODE_DIAG_SHIFT) & 7);
          const double res = (double)(a.sign * a.bdiv[q0 + L]) - (diag * s_x64[L] - sum);
          rf = (float)res;
          s_r[L] = rf;
          s_zb[tl * 1000 + pc] =
              SGS ? rf * s_rtab[8 | ((code >> CODE_DIAG_SHIFT) & 7)] : rf / diagz_of(code);
          vr[0] += res * res;
        }
        if (CRS && coarse && tl < nt) tile_partial(tl, rf);
      }
      if (SGS) zero_rings();
      double tr[1];
      if (!grid_allreduce<double, 1>(gs, vr, tr, shd)) return;
      r_true2 = tr[0];
      // z = M r from the replaced residuals (ring included), then w = A z
      precond_exchange();
      Acc vw[3] = {0, 0, 0};
#pragma unroll
      for (int j = 0; j < MAXJ; ++j) {
        if (!((fmask >> j) & 1)) continue;
        const int L = (tl0 + 2 * j) * 512 + l;
        float z;
        const float wn = stencil(j, z);
        const float r = s_r[L];
        s_w[L] = wn;
        vw[0] += (Acc)(r * z);
        vw[1] += (Acc)(wn * z);
        vw[2] += (Acc)(r * r);
      }
      if (!fast_allreduce3<Acc>(fs, gs, vw, tv, sh)) return;
      ++nrep;
      r_upd2 = (double)tv[2];
      rr_last = r_upd2;
      if (r_true2 <= a.tol2 * b2) done = 1;
    }
    // ---- scalars of the next iteration (Chronopoulos-Gear)
    // (beta' gamma' / alpha formed as gamma'^2 / (gamma alpha), so that its
    // division does not wait for beta's: two dependent divisions, not three)
    const Acc gamma_new = tv[0], delta = tv[1];
    const bool g_zero = fabs((double)gamma) < 1.0e-30;
    const Acc bnew = g_zero ? (Acc)0 : gamma_new / gamma;
    const Acc den = delta - (g_zero || fabs((double)alpha) < 1.0e-30
                                 ? (Acc)0
                                 : (Acc)((double)gamma_new * (double)gamma_new /
                                         ((double)gamma * (double)alpha)));
    alpha = fabs((double)den) < 1.0e-30 ? (Acc)0 : gamma_new / den;
    beta = bnew;
    gamma = gamma_new;
  }
  // ---- results
#pragma unroll
  for (int j = 0; j < MAXJ; ++j) {
    const int tl = tl0 + 2 * j;
    if (tl >= nt) break;
    const int L = tl * 512 + l;
    a.xf[q0 + L] = s_x[L];
    if (REF) a.x64[q0 + L] = s_x64[L];
  }
  if (gs.trace) {  // per block: busy cycles, tiles, fluid cells, remote faces
    __shared__ int s_nf;
    if (threadIdx.x == 0) s_nf = 0;
    __syncthreads();
    atomicAdd(&s_nf, __popc(fmask));
    __syncthreads();
    if (threadIdx.x == 0) {
      int remote = 0;
      for (int f = 0; f < nt * 6; ++f)
        if (s_nbr[f] >= 0 && !(s_nbr[f] >= b0 && s_nbr[f] < b1)) ++remote;
      long long *t = gs.trace + a.trace_cap / 2 + 12 * blockIdx.x;
      t[0] = gs.busy;
      t[1] = nt;
      t[2] = s_nf;
      t[3] = remote;
      for (int k = 0; k < 8; ++k) t[4 + k] = s_ph[k];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->trace_n = gs.trace_n;
    st->iters = iters;
    st->r0 = (double)r0;
    st->rr = rr_last;
    st->b2 = b2;
    st->r_true2 = r_true2;
    st->n_replace = nrep;
    st->done = done;
    st->status = done ? status : GF_NOT_CONVERGED;
    if (status != GF_OK) st->status = status;
    st->smem_solver = 1;
    st->coarse_used = coarse ? 1 : 0;
  }
}

template <typename Acc, bool REF>
static bool fits_t(Ctx *c) {
  int optin = 0;
  cudaFuncAttributes fa;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) !=
          cudaSuccess ||
      cudaFuncGetAttributes(&fa, (const void *)k_pcg_smem<Acc, REF, true, true>) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return SmemCfg<REF>::BYTES + fa.sharedSizeBytes <= (size_t)optin;
}

bool pcg_smem_fits(Ctx *c, bool refined) {
  return refined ? fits_t<double, true>(c) : fits_t<float, false>(c);
}

template <typename Acc, bool REF>
static int launch_t(Ctx *c, PcgSmemArgs &a) {
  const size_t smem = SmemCfg<REF>::BYTES;
  auto fn = a.sgs_sweeps > 0 ? (a.coarse ? k_pcg_smem<Acc, REF, true, true>
                                         : k_pcg_smem<Acc, REF, true, false>)
                             : (a.coarse ? k_pcg_smem<Acc, REF, false, true>
                                         : k_pcg_smem<Acc, REF, false, false>);
  int e = check_cuda(c, cudaFuncSetAttribute((const void *)fn,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem),
                     "PCG shared-memory size");
  if (e) return e;
  int per_sm = 0;
  e = check_cuda(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, SM_THREADS, smem),
                 "PCG occupancy");
  if (e) return e;
  if (per_sm < 1) return fail(c, GF_CUDA_ERROR, "PCG shared-memory kernel does not fit an SM");
  if (a.coarse && a.cbuf) {  // rows of A_c, then of B = A_c^-1, for the active tiles
    if ((e = coarse_setup_tiles(c, a.n_active, a.tile_list, a.nbr, a.code, a.st,
                                c->num_sms * SmemCfg<REF>::MAXT)))
      return e;
  }
  void *args[] = {&a};
  e = check_cuda(c, cudaLaunchCooperativeKernel((const void *)fn, dim3(c->num_sms),
                                                dim3(SM_THREADS), args, smem, c->stream),
                 "cooperative shared-memory PCG launch");
  c->launches++;
  return e;
}

int launch_pcg_smem(Ctx *c, PcgSmemArgs &a, bool refined) {
  return refined ? launch_t<double, true>(c, a) : launch_t<float, false>(c, a);
}

}  // namespace gf
