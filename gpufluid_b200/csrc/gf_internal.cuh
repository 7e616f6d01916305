// Internal declarations shared by the gfb200 translation units.
//
// Data layout in HBM (all device buffers):
//  * dense MAC fields exactly as the reference lays them out (C order, k
//    fastest), so the caller can hand in / read back the same arrays;
//  * labels as uint8 (0 air, 1 fluid, 2 solid): 1 B per cell instead of the
//    reference's int32 marker;
//  * particles in the caller's (n,3) AoS buffers hold the state between
//    substeps; inside a substep they are read from four float4 streams,
//    sorted by cell:  rec0 = (x, y, z, pid-as-bits); FLIP/PIC rec1 = (vx, vy,
//    vz, 0); APIC one record per face component c: rec1 = (vx, C00, C01, C02),
//    rec2 = (vy, C10, C11, C12), rec3 = (vz, C20, C21, C22), so that a
//    component's scatter reads two records
//    (FLIP/PIC use rec0, rec1 only);
//  * the pressure solve works on a compact array of active 8x8x8 tiles:
//    element (slot*512 + ((li*8 + lj)*8 + lk)) is cell (8*ti+li, 8*tj+lj,
//    8*tk+lk) of the slot-th active tile, with a 6-neighbour tile table and a
//    16-bit stencil code per cell.
#pragma once

#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point)
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/gfb200.h"

namespace gf {

constexpr int TILE = 8;            // tile edge in cells (the reference's BLOCK_SIZE, :950)
constexpr int TILE_CELLS = 512;    // cells per tile
constexpr int MAX_PCG_BLOCKS = 4096;
constexpr int COARSE_MAXG = 160;  // blocks of the shared-memory PCG, at most
// coarse regions (one per active tile of the shared-memory PCG), at most: 14
// tiles per block; a multiple of 8, so bf16 rows of this stride are 16-byte
// aligned
constexpr int COARSE_RMAX = COARSE_MAXG * 14;
static_assert(COARSE_RMAX % 8 == 0, "coarse row stride");
// coarse buffer: two sets of rows of B = (P^T A P)^-1 as bf16 [RMAX][RMAX]
// (the last solve's and the next), then the rows of P^T A P: diagonal [RMAX]
// and the six face-neighbour entries [RMAX][6] (floats), the tile of each row
// of the last B [RMAX] (ints), and CoarseMeta.  The meta and the tile-to-row
// map of the last B (Ctx::coarse_prev_slot) persist from solve to solve; the
// device keeps them, so CUDA-graph replays stay consistent.
constexpr int64_t COARSE_B_BYTES = (int64_t)COARSE_RMAX * COARSE_RMAX * 2;
struct CoarseMeta {
  int parity;   // which B set holds the last solve's rows
  int prev_na;  // rows of that B (0: none yet)
  int kind;     // COARSE_KIND_* of that B's regions
  int pad;
};
constexpr int COARSE_KIND_TILES = 0;    // one region per active tile (shared-memory PCG)
constexpr int COARSE_KIND_REGIONS = 1;  // cubes of RegionGrid::ct^3 tiles (global-memory PCG)
constexpr int COARSE_RG_DENSE_MAX = 8192;  // regions of the cube grid, at most

// The cube grid of the global-memory solver's coarse regions.
struct RegionGrid {
  int ct;             // tiles per region edge (a power of two)
  int nx, ny, nz, n;  // regions per axis, total
  int ntx, nty, ntz;  // tiles per axis
  __host__ __device__ int region_of_tile(int t) const {
    const int ti = t / (nty * ntz), tj = (t / ntz) % nty, tk = t % ntz;
    return ((ti / ct) * ny + tj / ct) * nz + tk / ct;
  }
};

struct PcgState;
// Arguments of the coarse set-up kernels (coarse.cu).
struct CoarseSetup {
  const int32_t *count;  // rows (device)
  const int32_t *ids;    // region id of each row: tile id or cube index
  const int32_t *nbr;    // [count][6] neighbouring rows, -1: none
  float *cdiag, *coff;   // rows of A_c: diagonal [RMAX], faces [RMAX][6]
  uint16_t *bsets;       // [2][RMAX][RMAX] bf16 rows of B
  int32_t *prev_slot;    // [ids] row of each id in the last B, or -1
  int32_t *prev_list;    // [RMAX] id of each row of the last B
  CoarseMeta *meta;
  PcgState *st;
  int limit;             // row counts above this skip the set-up
  const int *gate;       // nullable: the set-up runs only when *gate != 0
  int kind;              // COARSE_KIND_*
};
constexpr int64_t COARSE_DIAG_OFF = 2 * COARSE_B_BYTES;
constexpr int64_t COARSE_OFF_OFF = COARSE_DIAG_OFF + (int64_t)COARSE_RMAX * 4;
constexpr int64_t COARSE_LIST_OFF = COARSE_OFF_OFF + (int64_t)COARSE_RMAX * 6 * 4;
constexpr int64_t COARSE_META_OFF = COARSE_LIST_OFF + (int64_t)COARSE_RMAX * 4;
constexpr int64_t COARSE_BUF_BYTES = COARSE_META_OFF + (int64_t)sizeof(CoarseMeta);
constexpr int TRACE_CAP = 4096;
// Refined PCG: the FP64 residual replacement is taken each time the float32
// recursive residual fell by 100x (squared: 1e-4) since the last one.  1000x
// saved one replacement per 128^3 solve (2% of the solve) with the tile SGS
// preconditioner and the coarse correction, but with the Jacobi
// preconditioner the float32 recursion then stalls above the next threshold
// on harder systems (an 80^3 solve to 1e-10 ran out of iterations).
constexpr double PCG_REPLACE2 = 1e-4;

// Stencil code bits (per compact cell).
constexpr uint16_t CODE_NB_MASK = 0x3F;   // bit b: neighbour b is fluid (-x,+x,-y,+y,-z,+z)
constexpr int CODE_DIAG_SHIFT = 8;        // bits 8..10: #non-solid in-grid neighbours
constexpr uint16_t CODE_FLUID = 0x8000;   // the cell itself is fluid

struct PcgState {
  // scalars of the running solve (device resident)
  double rz;       // r . z
  double r0;       // ||r0||^2 (the reference's stop test base)
  double rr;       // ||r||^2 at the last evaluation
  double alpha, beta;
  double b2;       // ||b||^2 (refined solve)
  double r_true2;  // ||b - A x||^2 in FP64 at the last replacement
  double r_upd2;   // ||r||^2 at the last residual replacement
  int iters;
  int done;
  int status;      // gf_status
  int n_replace;   // residual replacements performed (refined solve)
  unsigned bar_count;
  unsigned bar_gen;
  int error;       // set on a barrier timeout
  int fallback;    // 1: the active region exceeded the shared-memory solver
  unsigned long long bar64;  // monotonic arrival counter (shared-memory solver)
  int smem_solver; // 1: the last solve ran in the shared-memory solver
  int trace_n;     // globaltimer stamps recorded (diagnostic trace)
  int coarse_off;  // a block's coarse-column solve failed: coarse correction off
  int coarse_used; // 1: the last solve applied the coarse correction
  double rz_part;  // global-memory solver with the coarse correction: r . M_tile r, before
                   // the coarse term r . P e is added
};

// Shared-memory-resident PCG (pcg_smem.cu).  Returns GF_OK after enqueuing;
// sets *launched to 1 when it was enqueued (it may still defer at run time to
// the global-memory solver through PcgState::fallback).
struct PcgSmemArgs {
  const int32_t *n_active, *nbr, *tile_cost;
  const uint16_t *code;
  const float *bdiv;
  float *xf;       // result (compact)
  float *hr0, *hr1, *hw0, *hw1, *hs0, *hs1;  // halo r, w, s by parity (compact index space)
  double *x64;     // refined: result and FP64 halo (compact)
  double *partials;  // [2][4][grid]
  unsigned long long *counter;  // barrier arrival counter (zeroed per solve)
  PcgState *st;
  long long *trace;  // nullable: per-phase globaltimer stamps of block 0
  int trace_cap;
  int max_iter, check_every;
  double tol2, replace2;
  float sign;
  int sgs_sweeps;             // 0: Jacobi (the reference's); 1-3: tile-local symmetric GS
  int coarse;                 // 1: tile coarse correction (one region per active tile)
  unsigned char *cbuf;        // coarse: bf16 rows of B, then the rows of P^T A P
  int test_stall;             // GF_FLAG_TEST_STALL: the first all-reduce waits for a count
                              // no block publishes, with a short spin limit
  // GF_FLAG_WARM_START (refined solve): start from the dense pressure p0 (the
  // previous substep's) instead of 0; tile_list and the grid shape map a
  // compact cell to its dense index
  int warm;
  const float *p0;
  const int32_t *tile_list;
  int ny, nz, nty, ntz;
};


// One scene of a batch (a row of the segment table, device resident).  The
// scenes' arrays are concatenated in table order: cells (labels, p, div),
// u-, v- and w-shaped faces, 8x8x8 tiles and sort keys, particles.
struct SegRow {
  int nx, ny, nz, ntx, nty, ntz;
  float dx, dom0, dom1, dom2;
  int64_t tile0;             // first global tile (key = tile * 512 + local cell)
  int64_t cell0;             // first cell
  int64_t fu0, fv0, fw0;     // first u, v, w face
  int64_t fslot0;            // first face slot ((nx+1)(ny+1)(nz+1) per scene)
};

// Prefix arrays of a batch for the scene lookup of a flat index (n+1 entries
// each, device resident).
struct SegIndex {
  const SegRow *row;
  const int64_t *tile0, *cell0, *fslot0, *part0;
  int n;
};

// Largest s with off[s] <= x (off ascending, off[0] = 0, n scenes).
__device__ __forceinline__ int seg_find(const int64_t *__restrict__ off, int n, int64_t x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(off + mid) <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// TMA descriptors of the six face arrays G2P stages per tile (u, v, w, us,
// vs, ws), encoded when the caller's buffers are bound.  Bit a of `mask` is
// set when array a's layout allows a tiled tensor map (16-byte aligned base
// and row / plane strides); G2P loads the other arrays' boxes with plain
// loads.
struct FaceMaps {
  CUtensorMap m[6];
  int mask;
};

// Launch shapes chosen by gf_autotune (defaults until it runs).
struct Tune {
  int p2g_tiles_k = 1;           // P2G and G2P blocks: 8 x 8 x 8 (1) or 8 x 8 x 16 cells (2)
  int g2p_tiles_k = 1;
  int p2g_map = 2;               // P2G lanes: runs of particles (0), one cell each (1), one
                                 // cell each summed in registers first (2)
  int g2p_threads = 256;
  int grid_threads = 256;        // forces / divergence / project / sweeps
  int grid_blocks_per_sm = 16;   // cap of their grid-stride launches
  int pcg_blocks_per_sm = 0;     // global-memory PCG: 0 = occupancy maximum
};

struct Ctx {
  // grid
  int nx = 0, ny = 0, nz = 0;
  float dx = 0.f, dom[3] = {0, 0, 0};
  int ntx = 0, nty = 0, ntz = 0, ntiles = 0;
  int64_t nkeys = 0;  // ntiles * 512
  int64_t ncell = 0;
  int device = 0, num_sms = 0;
  cudaStream_t stream = 0;

  // caller buffers
  gf_fields f{};
  gf_particles p{};
  FaceMaps face_maps{};   // tensor maps of the bound face arrays (single grid): 8^3 blocks
  FaceMaps face_maps2{};  // the same for 8 x 8 x 16 blocks (Tune::g2p_tiles_k = 2)
  // outflow compaction scratch (block counts, offsets, boxes), grown on use
  int32_t *region_scratch = nullptr;
  int64_t region_scratch_n = 0;
  bool bound = false;

  // binning scratch
  int64_t cap = 0;
  int32_t *key = nullptr, *rank = nullptr, *order = nullptr;
  int32_t *count = nullptr, *start = nullptr, *scan_part = nullptr;
  int64_t n_scan_blocks = 0;
  float4 *rec0 = nullptr, *rec1 = nullptr, *rec2 = nullptr, *rec3 = nullptr;

  // pressure workspace (compact active tiles)
  int32_t *tile_slot = nullptr;  // [ntiles] slot or -1
  int32_t *tile_list = nullptr;  // [ntiles] tile id of each slot
  int32_t *tile_order = nullptr; // [ntiles] Morton order of the tile ids (single grid)
  int32_t *tile_nbr = nullptr;   // [ntiles*6] neighbour slot or -1
  int32_t *n_active = nullptr;   // [0] active tiles, [1..2] fluid-cell count (int64)
  uint16_t *code = nullptr;      // [nkeys]
  float *bdiv = nullptr, *xf = nullptr, *r = nullptr, *z = nullptr;
  float *d0 = nullptr, *d1 = nullptr, *Ad = nullptr;
  double *x64 = nullptr;
  double *partials = nullptr;    // [3 * MAX_PCG_BLOCKS]
  unsigned long long *bar_counters = nullptr;  // 8 lines x 16 u64
  float *halo = nullptr;         // [6 * nkeys] halo publication buffers
  unsigned char *coarse_buf = nullptr;  // [COARSE_BUF_BYTES] coarse operator and inverse rows
  int32_t *coarse_prev_slot = nullptr;  // [max(ntiles, rg.n)] row of each id in the last B, or -1
  RegionGrid rg{};                      // coarse regions of the global-memory PCG
  int32_t *rg_buf = nullptr;            // region flags, slots, list, count, neighbours, tiles
  float *rg_gt = nullptr;               // [ntiles] residual sum of each tile slot (per iteration)
  float *rg_e = nullptr;                // [RMAX] coarse correction of each region (per iteration)
  int32_t *tile_cost = nullptr;  // [ntiles] per-slot PCG work estimate
  long long *trace = nullptr;    // [TRACE_CAP] PCG phase timestamps
  bool trace_on = false;
  PcgState *state = nullptr;
  PcgState *state_host = nullptr;  // pinned mirror
  // solve health since the last gf_health_read reset (device int32[8]):
  // [0] worst severity, [1] solves, [2] not converged, [3] failed, [4]
  // severity of the last call (folded in by the pressure scatter kernel),
  // [5] stage-kernel waits that ran out (the G2P tile loads)
  int32_t *health = nullptr;
  int last_solver = -1;  // gf_solver of the last gf_pressure
  int last_iters = 0;    // iteration count of the last Jacobi / GS-RB solve

  // adjoint workspace (allocated on the first gf_step_adjoint)
  float *adj_faces = nullptr;  // ubar3, qbar, mbar: 9 face arrays
  int64_t adj_faces_n = 0;
  float *adj_part = nullptr;   // per-particle position adjoint scratch
  int64_t adj_part_n = 0;

  // batch of scenes (nseg > 0): segment table and per-scene solve state
  int nseg = 0;
  SegRow *seg = nullptr;                 // [nseg]
  int64_t *seg_off = nullptr;            // 4 prefix arrays of nseg+1: tile0, cell0, fslot0, part0
  PcgState *seg_state = nullptr;         // [nseg]
  PcgState *seg_state_host = nullptr;    // pinned mirror
  int32_t *seg_slot0 = nullptr;          // [nseg+1] first active slot of each scene
  int32_t *pcg_blk_job0 = nullptr;       // [MAX_PCG_BLOCKS+1] segmented PCG: jobs per block
  void *pcg_jobs = nullptr;              // segmented PCG job table (pcg_jobs_bytes)
  int64_t nfslot = 0;                    // face slots of all scenes
  int64_t nu = 0, nv = 0, nw = 0;        // u, v, w faces of all scenes
  Tune tune;

  // diagnostics
  bool timing = false;
  cudaEvent_t ev[10] = {};  // 0..6 stage boundaries, 8..9 around the solver kernel
  int64_t launches = 0;
  float *vmax_dev = nullptr;
  std::string err;
};

// ---- bounds-checked build ---------------------------------------------------
// Built with -DGF_BOUNDS_CHECK (libgfb200_checked.so), GF_IN(i, n) checks
// 0 <= i < n for an index about to address global memory; a violation is
// counted in the translation unit's device counter (with the source line of
// the first one) and the access is skipped.  In the regular library GF_IN is
// `true` and compiles away.  Each instrumented file ends with
// GF_BOUNDS_READER(name), the host reader gf_bounds_status collects.
#ifdef GF_BOUNDS_CHECK
static __device__ unsigned long long g_bounds_hits;
static __device__ int g_bounds_line;
__device__ __forceinline__ bool gf_in(int64_t i, int64_t n, int line) {
  if (i >= 0 && i < n) return true;
  if (atomicAdd(&g_bounds_hits, 1ull) == 0ull) g_bounds_line = line;
  return false;
}
#define GF_IN(i, n) ::gf::gf_in((int64_t)(i), (int64_t)(n), __LINE__)
#define GF_BOUNDS_READER(name)                                                          \
  int bounds_read_##name(unsigned long long *hits, int *line, int reset) {             \
    if (cudaMemcpyFromSymbol(hits, g_bounds_hits, sizeof(*hits)) != cudaSuccess ||     \
        cudaMemcpyFromSymbol(line, g_bounds_line, sizeof(*line)) != cudaSuccess)        \
      return GF_CUDA_ERROR;                                                              \
    if (reset) {                                                                         \
      const unsigned long long z = 0;                                                    \
      if (cudaMemcpyToSymbol(g_bounds_hits, &z, sizeof(z)) != cudaSuccess)               \
        return GF_CUDA_ERROR;                                                            \
    }                                                                                    \
    return GF_OK;                                                                        \
  }
#else
#define GF_IN(i, n) true
#define GF_BOUNDS_READER(name)                                                          \
  int bounds_read_##name(unsigned long long *hits, int *line, int) {                   \
    *hits = 0;                                                                           \
    *line = 0;                                                                           \
    return GF_OK;                                                                        \
  }
#endif
int bounds_read_transfer(unsigned long long *hits, int *line, int reset);
int bounds_read_bin(unsigned long long *hits, int *line, int reset);
int bounds_read_pressure(unsigned long long *hits, int *line, int reset);

// ---- helpers ---------------------------------------------------------------
int fail(Ctx *c, int status, const std::string &msg);
int check_cuda(Ctx *c, cudaError_t e, const char *what);
int coarse_setup_tiles(Ctx *c, const int32_t *n_active, const int32_t *tile_list,
                       const int32_t *tile_nbr, const uint16_t *code, PcgState *st, int limit);
int coarse_setup_regions(Ctx *c, PcgState *st, const int *gate);
// Ctx::rg_buf: region flags and slots [rg.n], the active regions' list
// [RMAX], their count, neighbours [RMAX][6], tile slots [RMAX][ct^3] and the
// region of each tile slot [ntiles]
struct RegionBufs {
  int32_t *flag, *slot, *list, *count, *nbr, *tiles, *of_slot;
};
RegionBufs region_bufs(Ctx *c);
int check_launch(Ctx *c, const char *what);

// Packed float32 pairs (the sm_100 f32x2 instructions): one instruction does
// the operation on both halves.  mul2 / add2 / sub2 round each half exactly as
// the scalar IEEE operation (.rn), so a paired product or sum is bit-identical
// to the two scalar ones; fma2 fuses each half's multiply-add.
__device__ __forceinline__ unsigned long long f2_bits(const float2 &a) {
  return reinterpret_cast<const unsigned long long &>(a);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
  float2 d;
  asm("mul.rn.f32x2 %0, %1, %2;"
      : "=l"(reinterpret_cast<unsigned long long &>(d))
      : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return d;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
  float2 d;
  asm("add.rn.f32x2 %0, %1, %2;"
      : "=l"(reinterpret_cast<unsigned long long &>(d))
      : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  float2 d;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(reinterpret_cast<unsigned long long &>(d))
      : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return d;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  float2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(reinterpret_cast<unsigned long long &>(d))
      : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return d;
}
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
// x + y as fma(x, one, y), where `one` is 1 but known only at run time (a
// launch argument): x * 1 is exact, so the result is the correctly rounded
// sum of mul2 / add2, yet the compiler cannot merge a paired product that
// feeds it into a fused multiply-add.  (ptxas contracts mul.rn.f32x2 into a
// following add.rn.f32x2 even under --fmad=false; bit-exact code forms every
// paired sum of a product this way.)
__device__ __forceinline__ float2 sum2(float2 x, float2 one, float2 y) { return fma2(x, one, y); }

// 1/dx when dx is a power of two, so that x * (1/dx) is x / dx exactly; 0
// otherwise (the IEEE division is used then).
__host__ __device__ inline float exact_inverse(float dx) {
  int e;
  return (dx > 0.f && frexpf(dx, &e) == 0.5f) ? 1.0f / dx : 0.0f;
}
// x / dx rounded as the IEEE division: a product when inv (exact_inverse(dx))
// is non-zero.
__device__ __forceinline__ float div_dx(float x, float dx, float inv) {
  return inv != 0.0f ? x * inv : __fdiv_rn(x, dx);
}

// Cell (li * 8 + lj) * 8 + lk of colour c ((li + lj + lk) & 1 == c) that
// thread k (0..255) of a red-black half-sweep updates.  Warp w = k >> 5 takes
// planes li = (w & 3) + {0, 4}, rows lj = 2 (w >> 2) + {0, 1, 4, 5} and the
// four cells of the colour in each row, so that in a 10^3 padded box (plane
// pitch 100, row pitch 10) the warp's 32 cells -- and each of their six
// neighbours -- fall in 32 distinct shared-memory banks.
__device__ __forceinline__ int sgs_color_cell(int k, int c) {
  const int w = k >> 5, ln = k & 31, b = (ln >> 2) & 3;
  const int li = (w & 3) + 4 * (ln >> 4);
  const int lj = 2 * (w >> 2) + (b & 1) + 4 * (b >> 1);
  const int lk = 2 * (ln & 3) + ((li + lj + c) & 1);
  return (li * 8 + lj) * 8 + lk;
}

__host__ __device__ inline int64_t uidx(int i, int j, int k, int ny, int nz) {
  return ((int64_t)i * ny + j) * nz + k;
}

// Stage launchers (defined in the .cu files).
int launch_bin(Ctx *c, int transfer);
int launch_p2g(Ctx *c, int transfer);
int launch_forces_div(Ctx *c, float gravity, float dt, float rho);
int launch_pressure(Ctx *c, const gf_step_params *prm);
int launch_project(Ctx *c, float dt, float rho);
int launch_g2p(Ctx *c, int transfer, float flip_blend, float dt);
int launch_vmax(Ctx *c);
int encode_face_maps(Ctx *c);

int launch_pcg_smem(Ctx *c, PcgSmemArgs &a, bool refined);
bool pcg_smem_fits(Ctx *c, bool refined);

SegIndex seg_index(const Ctx *c);
size_t pcg_jobs_bytes(int nseg);

int pressure_alloc(Ctx *c);
void pressure_free(Ctx *c);

}  // namespace gf
