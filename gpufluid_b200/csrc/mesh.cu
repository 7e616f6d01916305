// Particles -> surface mesh, once per frame after the substeps
// (MeshExtractor.extract, src/gpufluid/meshing/surface.py:353-461).
//
// A mesher owns two density fields of the grid's cell count and the
// extraction scratch, like MeshExtractor's dens / dens_tmp (surface.py:
// 206-216).  gf_mesher_density builds the field:
//   k_mesh_zero + k_mesh_splat     trilinear unit-mass splat of each particle
//                                  (k_density_scatter, surface.py:14-43)
//   k_mesh_cubic                   or the cubic-falloff splat over a box of
//                                  cells (k_cubic_scatter, surface.py:53-84)
//   k_mesh_blur x smooth_passes    3x3x3 boundary-aware box blur
//                                  (k_box_blur_3d, gridmath.py:103-121); the
//                                  last pass also zeroes the wall margin
//   k_mesh_walls                   (k_mc_zero_walls, surface.py:179-193) when
//                                  there is no blur pass to fold it into
//   k_sdf_init/_scatter/_finish    or the signed distance to the nearest
//                                  particle (k_sdf_field, surface.py:100-122)
// The splats add with float atomics in arrival order (as the reference's
// wp.atomic_add); blur and margin are per-cell and follow the reference's
// float32 operation order exactly.
//
// gf_mesher_extract cuts the iso-surface density >= iso_level out of the field
// sampled at the cell indices (vertices are index * dx, as the reference's
// marching cubes returns them).  The reference hands this step to
// scikit-image's or Warp's marching cubes (surface.py:286-351).  This library
// writes its own, two ways (gf_mesher_set_surface):
//  * marching cubes (the default; Lorensen & Cline 1987).  A vertex sits on
//    each axis edge whose end values straddle the level, at the linear
//    crossing from the lower end.  The triangles of a cube come from a case
//    table this file generates (build_mc_table): on each cube face the
//    crossing edges pair into segments -- on an ambiguous face (two diagonal
//    corners inside, two outside) the pairs cut off the inside corners, so the
//    inside corners are never joined across a face.  That rule depends on the
//    face alone, so two cubes sharing a face cut it the same way and the
//    surface is closed wherever it does not meet the grid boundary.  The
//    segments chain into loops around the cube; each is oriented with the
//    inside on its right as seen from outside the cube, which makes every
//    triangle face from >= iso to < iso, listed from its lowest edge, and
//    fanned from its first vertex whose diagonals all leave the cube's faces
//    (a diagonal inside a face would meet the neighbouring cube's).  At most
//    5 triangles per cube.
//  * marching tetrahedra on the Kuhn (Freudenthal) split of every cube into
//    the six tetrahedra that share its main diagonal: conforming between
//    cubes, no ambiguous cases, no table.  Vertices also sit on the face
//    diagonals and the main diagonal (offsets from a node's lower corner); its
//    axis-edge vertices are the marching-cubes ones.
// Output order is fixed: vertices by (node, edge family), triangles by (cube,
// table entry or tet), so the mesh is deterministic for a given field.
//   k_mesh_count  per node: crossing-edge mask, cube corner mask, block sums
//   k_mesh_scan   block sums -> block offsets and the two totals (int64)
//   (host reads the totals, grows the output buffers)
//   k_mesh_vemit  per node: vertex ids and positions
//   k_mesh_temit  per cube: triangles (vertex ids looked up by edge owner)
#include <cuda_runtime.h>

#include <cub/cub.cuh>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/gfb200.h"

namespace gfm {

constexpr int MB = 256;        // threads per node block
constexpr int SCAN_T = 1024;   // threads of the offsets scan

struct Mesher {
  int nx = 0, ny = 0, nz = 0;
  float dx = 0.f;
  int64_t nnode = 0;
  int nb = 0;  // node blocks
  cudaStream_t stream = 0;
  float *dens = nullptr, *tmp = nullptr;
  uint8_t *vmask = nullptr, *cmask = nullptr;
  int32_t *vbase = nullptr;
  int64_t *sums = nullptr;     // [2 nb] block sums (verts, tris), [2 nb] offsets, [2] totals
  int64_t *tot_host = nullptr; // pinned [2]
  float *verts = nullptr;
  int64_t verts_cap = 0;
  int32_t *tris = nullptr;
  int64_t tris_cap = 0;
  int64_t nv = -1, nt = -1;    // counts of the last extraction
  int below = 0;               // 1: the surface encloses field <= iso (signed distances)
  int surface = GF_SURFACE_MARCHING_CUBES;
  int64_t launches = 0;
  // mesh smoothing scratch, grown on use
  void *sm_buf = nullptr;
  size_t sm_cap = 0;
  std::string err;
};

static int fail(Mesher *m, int status, const std::string &msg) {
  if (m) m->err = msg;
  return status;
}

static int check(Mesher *m, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return GF_OK;
  return fail(m, GF_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---- density field ---------------------------------------------------------
__global__ void k_mesh_zero(float *d, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) d[i] = 0.f;
}

// k_density_scatter: corner weights (1-s | s) per axis, w = wx * wy * wz.
__global__ void k_mesh_splat(const float *__restrict__ pos, int64_t n, float dx, int nx, int ny,
                             int nz, float *dens) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float fx = __fdiv_rn(pos[3 * q], dx) - 0.5f;
  const float fy = __fdiv_rn(pos[3 * q + 1], dx) - 0.5f;
  const float fz = __fdiv_rn(pos[3 * q + 2], dx) - 0.5f;
  const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
            k0 = __float2int_rz(floorf(fz));
  const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int ii = i0 + a, jj = j0 + b, kk = k0 + e;
        if (ii >= 0 && ii < nx && jj >= 0 && jj < ny && kk >= 0 && kk < nz)
          atomicAdd(&dens[((int64_t)ii * ny + jj) * nz + kk], wx[a] * wy[b] * wz[e]);
      }
}

// k_cubic_scatter: (1 - r^2)^3 for r^2 = |cell centre - p|^2 / R^2 < 1 over the
// cells within half_cells of the particle's lower trilinear corner.
__global__ void k_mesh_cubic(const float *__restrict__ pos, int64_t n, float dx,
                             float inv_r_world_sq, int half_cells, int nx, int ny, int nz,
                             float *dens) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float p0 = pos[3 * q], p1 = pos[3 * q + 1], p2 = pos[3 * q + 2];
  const int cx = __float2int_rz(floorf(__fdiv_rn(p0, dx) - 0.5f));
  const int cy = __float2int_rz(floorf(__fdiv_rn(p1, dx) - 0.5f));
  const int cz = __float2int_rz(floorf(__fdiv_rn(p2, dx) - 0.5f));
  const int ilo = max(0, cx - half_cells), ihi = min(nx, cx + half_cells + 1);
  const int jlo = max(0, cy - half_cells), jhi = min(ny, cy + half_cells + 1);
  const int klo = max(0, cz - half_cells), khi = min(nz, cz + half_cells + 1);
  for (int i = ilo; i < ihi; ++i) {
    const float ddx = ((float)i + 0.5f) * dx - p0;
    for (int j = jlo; j < jhi; ++j) {
      const float ddy = ((float)j + 0.5f) * dx - p1;
      for (int k = klo; k < khi; ++k) {
        const float ddz = ((float)k + 0.5f) * dx - p2;
        const float r_sq = (ddx * ddx + ddy * ddy + ddz * ddz) * inv_r_world_sq;
        if (r_sq < 1.0f) {
          const float om = 1.0f - r_sq;
          atomicAdd(&dens[((int64_t)i * ny + j) * nz + k], om * om * om);
        }
      }
    }
  }
}

__device__ __forceinline__ bool in_margin(int i, int j, int k, int nx, int ny, int nz, int m) {
  return i < m || i >= nx - m || j < m || j >= ny - m || k < m || k >= nz - m;
}

// k_box_blur_3d: sum of the in-grid 3x3x3 neighbours (di, dj, dk ascending,
// float32 adds in that order) divided by their count.  margin > 0 writes 0
// inside the wall margin instead (k_mc_zero_walls after the last pass).
__global__ void k_mesh_blur(const float *__restrict__ src, float *__restrict__ dst, int nx,
                            int ny, int nz, int margin) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz) return;
  const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((int64_t)ny * nz));
  if (margin > 0 && in_margin(i, j, k, nx, ny, nz, margin)) {
    dst[c] = 0.f;
    return;
  }
  float s = 0.f, cnt = 0.f;
  for (int di = -1; di <= 1; ++di) {
    const int ii = i + di;
    if (ii < 0 || ii >= nx) continue;
    for (int dj = -1; dj <= 1; ++dj) {
      const int jj = j + dj;
      if (jj < 0 || jj >= ny) continue;
      const float *row = src + ((int64_t)ii * ny + jj) * nz;
      for (int dk = -1; dk <= 1; ++dk) {
        const int kk = k + dk;
        if (kk < 0 || kk >= nz) continue;
        s = __fadd_rn(s, __ldg(row + kk));
        cnt += 1.0f;
      }
    }
  }
  dst[c] = __fdiv_rn(s, cnt);
}

__global__ void k_mesh_walls(float *d, int nx, int ny, int nz, int margin) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz) return;
  const int k = (int)(c % nz), j = (int)((c / nz) % ny), i = (int)(c / ((int64_t)ny * nz));
  if (in_margin(i, j, k, nx, ny, nz, margin)) d[c] = 0.f;
}

// k_sdf_field (surface.py:100-122): phi = sqrt(min(R^2, nearest d^2)) - r over
// the cell centres; the reference asks a hash grid for every cell's
// candidates, here every particle lowers the squared distance of the cells
// around it (an atomic minimum on the float's bits, which order like the
// non-negative floats).  d = centre - p, d^2 = (dx dx + dy dy) + dz dz.
__global__ void k_sdf_init(unsigned *bits, int64_t n, float r2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) bits[i] = __float_as_uint(r2);
}

__global__ void k_sdf_scatter(const float *__restrict__ pos, int64_t n, float dx, float R,
                              float r2, int nx, int ny, int nz, unsigned *bits) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float p[3] = {pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]};
  const int dims[3] = {nx, ny, nz};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {  // cells whose centre may lie within R, one cell of margin
    lo[a] = max(0, __float2int_rd(__fdiv_rn(p[a] - R, dx) - 0.5f) - 1);
    hi[a] = min(dims[a] - 1, __float2int_rd(__fdiv_rn(p[a] + R, dx) - 0.5f) + 1);
  }
  for (int i = lo[0]; i <= hi[0]; ++i) {
    const float ddx = ((float)i + 0.5f) * dx - p[0];
    for (int j = lo[1]; j <= hi[1]; ++j) {
      const float ddy = ((float)j + 0.5f) * dx - p[1];
      const float sxy = ddx * ddx + ddy * ddy;
      if (!(sxy < r2)) continue;
      for (int k = lo[2]; k <= hi[2]; ++k) {
        const float ddz = ((float)k + 0.5f) * dx - p[2];
        const float d2 = sxy + ddz * ddz;
        if (!(d2 < r2)) continue;
        unsigned *b = bits + ((int64_t)i * ny + j) * nz + k;
        const unsigned v = __float_as_uint(d2);
        if (v < *b) atomicMin(b, v);
      }
    }
  }
}

__global__ void k_sdf_finish(float *phi, int64_t n, float r) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) phi[i] = __fsqrt_rn(phi[i]) - r;  // phi holds the minimum's bits
}

// ---- iso-surface -----------------------------------------------------------
// Corner b of a cube (bit 0: +x, bit 1: +y, bit 2: +z) sits at node
// n + off(b).  Edge family b (1..7) of a node joins it to n + off(b).
// Tet t of the Kuhn split visits corners 0, a, a|b', 7 for the axis order
// (a, b', c) of permutation t; its orientation sign is the permutation's.
__constant__ uint8_t c_perm[6][2] = {{1, 2}, {1, 4}, {2, 1}, {2, 4}, {4, 1}, {4, 2}};
__constant__ int8_t c_parity[6] = {1, -1, -1, 1, 1, -1};

__device__ __forceinline__ void tet_corners(int t, int cs[4]) {
  cs[0] = 0;
  cs[1] = c_perm[t][0];
  cs[2] = c_perm[t][0] | c_perm[t][1];
  cs[3] = 7;
}

__device__ __forceinline__ int tet_tris(int in4) {
  const int c = __popc(in4);
  return (c == 1 || c == 3) ? 1 : (c == 2 ? 2 : 0);
}

__device__ __forceinline__ int cube_tris(int cm) {
  int s = 0;
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    int cs[4];
    tet_corners(t, cs);
    int in4 = 0;
#pragma unroll
    for (int v = 0; v < 4; ++v) in4 |= ((cm >> cs[v]) & 1) << v;
    s += tet_tris(in4);
  }
  return s;
}

// ---- marching-cubes case table ----------------------------------------------
// Edge e of a cube runs along axis bit a = 1, 2, 4 for e / 4 = 0, 1, 2, from
// corner lo, the (e % 4)-th corner (ascending) without bit a, to lo | a.
// Case cm (bit c: corner c is inside) has c_mc_ntri[cm] triangles, edges
// c_mc_tri[cm][3 t + 0..2].
struct McTable {
  uint8_t edge[12][2];
  uint8_t ntri[256];
  uint8_t tri[256][15];
};
__constant__ McTable c_mc;

static McTable build_mc_table() {
  McTable t{};
  int ne = 0;
  for (int a = 1; a <= 4; a <<= 1)
    for (int lo = 0; lo < 8; ++lo)
      if (!(lo & a)) {
        t.edge[ne][0] = (uint8_t)lo;
        t.edge[ne][1] = (uint8_t)(lo | a);
        ++ne;
      }
  // doubled coordinates: corner c at 2 * bits, an edge's midpoint at the sum
  auto cc = [](int c, int k) { return 2 * ((c >> k) & 1); };
  for (int cm = 0; cm < 256; ++cm) {
    auto in = [&](int c) { return (cm >> c) & 1; };
    int next[12];
    bool cross[12];
    for (int e = 0; e < 12; ++e) {
      next[e] = -1;
      cross[e] = in(t.edge[e][0]) != in(t.edge[e][1]);
    }
    for (int k = 0; k < 3; ++k)
      for (int side = 0; side < 2; ++side) {
        const int a = 1 << k, sv = side ? a : 0;
        int fe[4], nf = 0;  // crossing edges of the face
        for (int e = 0; e < 12; ++e)
          if ((t.edge[e][0] & a) == sv && (t.edge[e][1] & a) == sv && cross[e]) fe[nf++] = e;
        int pairs[2][2], np = 0;
        if (nf == 2) {
          pairs[0][0] = fe[0];
          pairs[0][1] = fe[1];
          np = 1;
        } else if (nf == 4) {  // ambiguous face: cut off each inside corner
          for (int c = 0; c < 8; ++c) {
            if ((c & a) != sv || !in(c)) continue;
            int m = 0;
            for (int q = 0; q < 4; ++q)
              if (t.edge[fe[q]][0] == c || t.edge[fe[q]][1] == c) pairs[np][m++] = fe[q];
            ++np;
          }
        }
        for (int q = 0; q < np; ++q) {
          const int e1 = pairs[q][0], e2 = pairs[q][1];
          int m1[3], m2[3], n[3] = {0, 0, 0}, w[3];
          const int cin = in(t.edge[e1][0]) ? t.edge[e1][0] : t.edge[e1][1];
          for (int d = 0; d < 3; ++d) {
            m1[d] = cc(t.edge[e1][0], d) + cc(t.edge[e1][1], d);
            m2[d] = cc(t.edge[e2][0], d) + cc(t.edge[e2][1], d);
            w[d] = 2 * cc(cin, d) - m1[d];
          }
          n[k] = side ? 1 : -1;  // the face's outward normal
          const int dv[3] = {m2[0] - m1[0], m2[1] - m1[1], m2[2] - m1[2]};
          const int lx = n[1] * dv[2] - n[2] * dv[1], ly = n[2] * dv[0] - n[0] * dv[2],
                    lz = n[0] * dv[1] - n[1] * dv[0];
          const bool left = lx * w[0] + ly * w[1] + lz * w[2] > 0;
          if (left)  // keep the inside on the right
            next[e2] = e1;
          else
            next[e1] = e2;
        }
      }
    // faces holding edge e: bit 2 k + side for the two faces off its axis
    auto fmask = [&](int e) {
      const int lo = t.edge[e][0], ax = t.edge[e][1] ^ lo;
      int m = 0;
      for (int k = 0; k < 3; ++k)
        if ((1 << k) != ax) m |= 1 << (2 * k + ((lo >> k) & 1));
      return m;
    };
    bool seen[12] = {};
    int nt = 0;
    for (int e0 = 0; e0 < 12; ++e0) {
      if (!cross[e0] || seen[e0]) continue;
      int loop[12], nl = 0;
      for (int e = e0; e >= 0 && !seen[e]; e = next[e]) {
        seen[e] = true;
        loop[nl++] = e;
      }
      // fan from the first vertex whose diagonals all leave the cube's faces:
      // a diagonal inside a face would meet the neighbouring cube's
      int s0 = 0;
      for (int k = 0; k < nl; ++k) {
        bool ok = true;
        for (int q = 2; q + 1 < nl; ++q) ok = ok && !(fmask(loop[k]) & fmask(loop[(k + q) % nl]));
        if (ok) {
          s0 = k;
          break;
        }
      }
      for (int q = 1; q + 1 < nl; ++q) {
        t.tri[cm][3 * nt] = (uint8_t)loop[s0];
        t.tri[cm][3 * nt + 1] = (uint8_t)loop[(s0 + q) % nl];
        t.tri[cm][3 * nt + 2] = (uint8_t)loop[(s0 + q + 1) % nl];
        ++nt;
      }
    }
    t.ntri[cm] = (uint8_t)nt;
  }
  return t;
}

struct NodeIdx {
  int i, j, k;
};

__device__ __forceinline__ NodeIdx node_of(int64_t n, int ny, int nz) {
  return {(int)(n / ((int64_t)ny * nz)), (int)((n / nz) % ny), (int)(n % nz)};
}

__device__ __forceinline__ int64_t off_of(int b, int ny, int nz) {
  return (b & 1 ? (int64_t)ny * nz : 0) + (b & 2 ? nz : 0) + (b & 4 ? 1 : 0);
}

// Block-wide exclusive prefix of v (MB threads); *total gets the block sum.
__device__ __forceinline__ int block_prefix(int v, int *total) {
  __shared__ int ws[MB / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < MB / 32; ++w) {
    const int s = ws[w];
    before += w < wid ? s : 0;
    all += s;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

struct ExtractArgs {
  const float *dens;
  float iso;
  int below;  // inside = value <= iso instead of >= iso
  int mc;     // 1: marching cubes (axis-edge vertices, table triangles)
  int nx, ny, nz;
  int64_t nnode;
  float dx;
  uint8_t *vmask, *cmask;
  int32_t *vbase;
  int64_t *sums;  // block sums v [nb], t [nb]; offsets v [nb], t [nb]; totals [2]
  int nb;
  float *verts;
  int32_t *tris;
};

__global__ void __launch_bounds__(MB) k_mesh_count(ExtractArgs a) {
  const int64_t n = blockIdx.x * (int64_t)MB + threadIdx.x;
  int vm = 0, cm = 0, nt = 0;
  if (n < a.nnode) {
    const NodeIdx p = node_of(n, a.ny, a.nz);
    const bool hx = p.i + 1 < a.nx, hy = p.j + 1 < a.ny, hz = p.k + 1 < a.nz;
    const float v0 = a.dens[n];
    const int in0 = a.below ? v0 <= a.iso : v0 >= a.iso;
    cm = in0;
#pragma unroll
    for (int b = 1; b < 8; ++b) {
      if ((b & 1 && !hx) || (b & 2 && !hy) || (b & 4 && !hz)) continue;
      const float vb = a.dens[n + off_of(b, a.ny, a.nz)];
      const int in = a.below ? vb <= a.iso : vb >= a.iso;
      cm |= in << b;
      if (!a.mc || b == 1 || b == 2 || b == 4) vm |= (in != in0) << b;
    }
    if (!(hx && hy && hz)) cm = 0;  // not the lower corner of a cube
    nt = (hx && hy && hz) ? (a.mc ? c_mc.ntri[cm] : cube_tris(cm)) : 0;
    a.vmask[n] = (uint8_t)vm;
    a.cmask[n] = (uint8_t)cm;
  }
  __shared__ int red[2][MB / 32];
  int sv = __popc(vm), st = nt;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sv += __shfl_down_sync(0xffffffffu, sv, o);
    st += __shfl_down_sync(0xffffffffu, st, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = sv;
    red[1][wid] = st;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t tv = 0, tt = 0;
    for (int w = 0; w < MB / 32; ++w) {
      tv += red[0][w];
      tt += red[1][w];
    }
    a.sums[blockIdx.x] = tv;
    a.sums[a.nb + blockIdx.x] = tt;
  }
}

// Exclusive offsets of the per-block sums; block 0 scans the vertex sums,
// block 1 the triangle sums, each in chunks of SCAN_T.
__global__ void __launch_bounds__(SCAN_T) k_mesh_scan(int64_t *sums, int nb) {
  __shared__ int64_t ws[SCAN_T / 32];
  __shared__ int64_t carry;
  const int64_t *in = sums + (int64_t)blockIdx.x * nb;
  int64_t *out = sums + 2 * (int64_t)nb + (int64_t)blockIdx.x * nb;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += SCAN_T) {
    const int t = base + threadIdx.x;
    const int64_t v = t < nb ? in[t] : 0;
    int64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const int64_t s = ws[lane];
      int64_t si = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t u = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += u;
      }
      ws[lane] = si - s;
    }
    __syncthreads();
    if (t < nb) out[t] = carry + ws[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == SCAN_T - 1) carry += ws[wid] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[4 * (int64_t)nb + blockIdx.x] = carry;
}

__global__ void __launch_bounds__(MB) k_mesh_vemit(ExtractArgs a) {
  const int64_t n = blockIdx.x * (int64_t)MB + threadIdx.x;
  const int vm = n < a.nnode ? a.vmask[n] : 0;
  int total;
  const int local = block_prefix(__popc(vm), &total);
  if (n >= a.nnode) return;
  const int64_t base = a.sums[2 * (int64_t)a.nb + blockIdx.x] + local;
  a.vbase[n] = (int32_t)base;
  if (!vm) return;
  const NodeIdx p = node_of(n, a.ny, a.nz);
  const float va = a.dens[n];
  const float fi = (float)p.i, fj = (float)p.j, fk = (float)p.k;
  int r = 0;
#pragma unroll
  for (int b = 1; b < 8; ++b) {
    if (!(vm >> b & 1)) continue;
    const float vb = a.dens[n + off_of(b, a.ny, a.nz)];
    const float t = __fdiv_rn(__fsub_rn(a.iso, va), __fsub_rn(vb, va));
    float *o = a.verts + 3 * (base + r);
    o[0] = __fmul_rn(b & 1 ? __fadd_rn(fi, t) : fi, a.dx);
    o[1] = __fmul_rn(b & 2 ? __fadd_rn(fj, t) : fj, a.dx);
    o[2] = __fmul_rn(b & 4 ? __fadd_rn(fk, t) : fk, a.dx);
    ++r;
  }
}

// Id of the vertex on the edge from cube corner lo to corner hi (lo's bits
// a subset of hi's): owned by node n + off(lo), family hi ^ lo.
__device__ __forceinline__ int32_t edge_vertex(const ExtractArgs &a, int64_t n, int lo, int hi) {
  const int64_t o = n + off_of(lo, a.ny, a.nz);
  const int f = hi ^ lo;
  return a.vbase[o] + __popc(a.vmask[o] & ((1 << f) - 1));
}

__global__ void __launch_bounds__(MB) k_mesh_temit(ExtractArgs a) {
  const int64_t n = blockIdx.x * (int64_t)MB + threadIdx.x;
  const int cm = n < a.nnode ? a.cmask[n] : 0;
  const int nt = (cm != 0 && cm != 0xff) ? (a.mc ? c_mc.ntri[cm] : cube_tris(cm)) : 0;
  int total;
  const int local = block_prefix(nt, &total);
  if (n >= a.nnode || nt == 0) return;
  int64_t w = a.sums[3 * (int64_t)a.nb + blockIdx.x] + local;
  if (a.mc) {
    int32_t *o = a.tris + 3 * w;
    for (int q = 0; q < 3 * nt; ++q) {
      const int e = c_mc.tri[cm][q];
      o[q] = edge_vertex(a, n, c_mc.edge[e][0], c_mc.edge[e][1]);
    }
    return;
  }
  for (int t = 0; t < 6; ++t) {
    int cs[4];
    tet_corners(t, cs);
    int in4 = 0;
#pragma unroll
    for (int v = 0; v < 4; ++v) in4 |= ((cm >> cs[v]) & 1) << v;
    const int cnt = __popc(in4);
    if (cnt == 0 || cnt == 4) continue;
    const int s = c_parity[t];
    int32_t *o = a.tris + 3 * w;
    if (cnt == 1 || cnt == 3) {
      // the lone vertex l and the others in ascending order: the triple
      // faces away from l when (-1)^l * s > 0; away is outward when l is
      // the inside vertex
      const int lone_in = cnt == 1;
      int l = 0;
      for (int v = 0; v < 4; ++v)
        if (((in4 >> v) & 1) == lone_in) l = v;
      int oth[3], m = 0;
      for (int v = 0; v < 4; ++v)
        if (v != l) oth[m++] = v;
      int32_t e[3];
      for (int q = 0; q < 3; ++q) {
        const int u = min(l, oth[q]), x = max(l, oth[q]);
        e[q] = edge_vertex(a, n, cs[u], cs[x]);
      }
      const bool away = ((l & 1) ? -s : s) > 0;
      o[0] = e[0];
      if (away == (bool)lone_in) {
        o[1] = e[1];
        o[2] = e[2];
      } else {
        o[1] = e[2];
        o[2] = e[1];
      }
      w += 1;
    } else {
      // inside pair (p0 < p1), outside pair (q0 < q1); the cycle
      // (p0q0, p0q1, p1q1, p1q0) faces outward when the tet reordered as
      // (p0, p1, q0, q1) is positive
      int pi[2], qo[2], np = 0, nq = 0;
      for (int v = 0; v < 4; ++v) {
        if ((in4 >> v) & 1)
          pi[np++] = v;
        else
          qo[nq++] = v;
      }
      const int ord[4] = {pi[0], pi[1], qo[0], qo[1]};
      int inv = 0;
      for (int x = 0; x < 4; ++x)
        for (int y = x + 1; y < 4; ++y) inv += ord[x] > ord[y];
      const int sp = (inv & 1) ? -s : s;
      auto E = [&](int u, int x) { return edge_vertex(a, n, cs[min(u, x)], cs[max(u, x)]); };
      int32_t cyc[4] = {E(pi[0], qo[0]), E(pi[0], qo[1]), E(pi[1], qo[1]), E(pi[1], qo[0])};
      if (sp < 0) {
        const int32_t tmp = cyc[1];
        cyc[1] = cyc[3];
        cyc[3] = tmp;
      }
      o[0] = cyc[0];
      o[1] = cyc[1];
      o[2] = cyc[2];
      o[3] = cyc[0];
      o[4] = cyc[2];
      o[5] = cyc[3];
      w += 2;
    }
  }
}

static int grow(Mesher *m, void **buf, int64_t *cap, int64_t need, int64_t elem,
                const char *what) {
  if (*cap >= need) return GF_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  const int64_t n = need + need / 4 + 1024;
  int e = check(m, cudaMalloc(buf, n * elem), what);
  if (e) return e;
  *cap = n;
  return GF_OK;
}

// ---- mesh smoothing (smoothing.py:22-72) ------------------------------------
// The uniform Laplacian L = D^-1 A - I of the triangles' 1-rings, A the
// 0/1 adjacency of distinct neighbours, D = diag(#neighbours) (1 for an
// isolated vertex).  The reference builds it with scipy in float64 from a
// float32 1/deg; a row of its CSR holds the diagonal first and then the
// neighbours in ascending order, and L @ v accumulates in that order from 0,
// a multiply and an add per entry.  Each pass replaces v by v + c (L v) in
// float64 (c = lam; Taubin adds a second step with c = mu); the result is
// rounded to float32 once at the end.  The adjacency: the 6 directed edges
// of every triangle as (row << 32 | col) keys, radix-sorted, deduplicated and
// counted per row into CSR offsets.
__global__ void k_edge_keys(const int32_t *__restrict__ tris, int64_t nt,
                            unsigned long long *keys) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const unsigned long long a = (unsigned)tris[3 * t], b = (unsigned)tris[3 * t + 1],
                           c = (unsigned)tris[3 * t + 2];
  unsigned long long *k = keys + 6 * t;
  k[0] = a << 32 | b;
  k[1] = b << 32 | a;
  k[2] = b << 32 | c;
  k[3] = c << 32 | b;
  k[4] = c << 32 | a;
  k[5] = a << 32 | c;
}

__global__ void k_row_counts(const unsigned long long *__restrict__ ukeys,
                             const int64_t *__restrict__ nu, int32_t *counts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= *nu) return;
  atomicAdd(&counts[(int64_t)(ukeys[i] >> 32)], 1);
}

__global__ void k_to_double(const float *__restrict__ v, int64_t n, double *d) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) d[i] = (double)v[i];
}

__global__ void k_to_float(const double *__restrict__ d, int64_t n, float *v) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) v[i] = (float)d[i];
}

// v_out = v_in + c (L v_in), one vertex per thread, the reference's order
__global__ void k_smooth_step(const double *__restrict__ vin, double *__restrict__ vout,
                              const int32_t *__restrict__ row, const unsigned long long *__restrict__ ukeys,
                              int64_t nv, double c) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nv) return;
  const int b = row[i], e = row[i + 1];
  const int deg = e - b;
  const double dinv = (double)__fdiv_rn(1.0f, (float)(deg > 0 ? deg : 1));
  double acc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) acc[k] = __dadd_rn(0.0, __dmul_rn(-1.0, vin[3 * i + k]));
  for (int q = b; q < e; ++q) {
    const int64_t j = (int64_t)(ukeys[q] & 0xffffffffull);
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = __dadd_rn(acc[k], __dmul_rn(dinv, vin[3 * j + k]));
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) vout[3 * i + k] = __dadd_rn(vin[3 * i + k], __dmul_rn(c, acc[k]));
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static int smooth(Mesher *m, float *verts, int64_t nv, const int32_t *tris, int64_t nt,
                  int method, int passes, double lam, double mu) {
  cudaStream_t st = m->stream;
  const int64_t ne = 6 * nt;
  // scratch: keys, sorted keys, unique keys, unique count, row offsets, two
  // double vertex buffers, CUB temporaries
  size_t tmp_sort = 0, tmp_uniq = 0, tmp_scan = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, tmp_sort, (unsigned long long *)nullptr,
                                 (unsigned long long *)nullptr, (int64_t)ne, 0, 64, st);
  cub::DeviceSelect::Unique(nullptr, tmp_uniq, (unsigned long long *)nullptr,
                            (unsigned long long *)nullptr, (int64_t *)nullptr, (int64_t)ne, st);
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, (int32_t *)nullptr, (int32_t *)nullptr,
                                (int64_t)(nv + 1), st);
  size_t tmp = tmp_sort > tmp_uniq ? tmp_sort : tmp_uniq;
  tmp = tmp > tmp_scan ? tmp : tmp_scan;
  const size_t o_k0 = 0, o_k1 = align256(o_k0 + ne * 8), o_nu = align256(o_k1 + ne * 8),
               o_cnt = align256(o_nu + 8), o_row = align256(o_cnt + (nv + 1) * 4),
               o_v0 = align256(o_row + (nv + 1) * 4),
               o_v1 = align256(o_v0 + nv * 24), o_tmp = align256(o_v1 + nv * 24),
               total = o_tmp + tmp;
  if (m->sm_cap < total) {
    if (m->sm_buf) cudaFree(m->sm_buf);
    m->sm_buf = nullptr;
    m->sm_cap = 0;
    int e = check(m, cudaMalloc(&m->sm_buf, total), "alloc smoothing scratch");
    if (e) return e;
    m->sm_cap = total;
  }
  char *base = reinterpret_cast<char *>(m->sm_buf);
  auto *k0 = reinterpret_cast<unsigned long long *>(base + o_k0);
  auto *k1 = reinterpret_cast<unsigned long long *>(base + o_k1);
  auto *nu = reinterpret_cast<int64_t *>(base + o_nu);
  auto *cnt = reinterpret_cast<int32_t *>(base + o_cnt);
  auto *row = reinterpret_cast<int32_t *>(base + o_row);
  auto *v0 = reinterpret_cast<double *>(base + o_v0);
  auto *v1 = reinterpret_cast<double *>(base + o_v1);
  void *cub_tmp = base + o_tmp;
  int e;
  const unsigned g_t = (unsigned)((nt + 255) / 256), g_e = (unsigned)((ne + 255) / 256),
                 g_v = (unsigned)((nv + 255) / 256), g_c = (unsigned)((3 * nv + 255) / 256);
  if (ne == 0) return fail(m, GF_INVALID_ARG, "gf_mesher_smooth: no triangles");
  k_edge_keys<<<g_t, 256, 0, st>>>(tris, nt, k0);
  size_t t1 = tmp;
  if ((e = check(m, cub::DeviceRadixSort::SortKeys(cub_tmp, t1, k0, k1, (int64_t)ne, 0, 64, st),
                 "sort edge keys")))
    return e;
  t1 = tmp;
  if ((e = check(m, cub::DeviceSelect::Unique(cub_tmp, t1, k1, k0, nu, (int64_t)ne, st),
                 "unique edge keys")))
    return e;
  if ((e = check(m, cudaMemsetAsync(cnt, 0, (nv + 1) * 4, st), "zero row counts"))) return e;
  k_row_counts<<<g_e, 256, 0, st>>>(k0, nu, cnt);
  t1 = tmp;
  if ((e = check(m, cub::DeviceScan::ExclusiveSum(cub_tmp, t1, cnt, row, (int64_t)(nv + 1), st),
                 "row offsets")))
    return e;
  k_to_double<<<g_c, 256, 0, st>>>(verts, 3 * nv, v0);
  m->launches += 4;
  double *a = v0, *b = v1;
  for (int p = 0; p < passes; ++p) {
    k_smooth_step<<<g_v, 256, 0, st>>>(a, b, row, k0, nv, lam);
    double *t = a;
    a = b;
    b = t;
    m->launches++;
    if (method == GF_MESH_SMOOTH_TAUBIN) {
      k_smooth_step<<<g_v, 256, 0, st>>>(a, b, row, k0, nv, mu);
      t = a;
      a = b;
      b = t;
      m->launches++;
    }
  }
  k_to_float<<<g_c, 256, 0, st>>>(a, 3 * nv, verts);
  m->launches++;
  return check(m, cudaGetLastError(), "mesh smoothing");
}

static void release(Mesher *m) {
  void *ps[] = {m->dens, m->tmp, m->vmask, m->cmask, m->vbase, m->sums, m->verts, m->tris,
                m->sm_buf};
  for (void *p : ps)
    if (p) cudaFree(p);
  if (m->tot_host) cudaFreeHost(m->tot_host);
}

}  // namespace gfm

using gfm::Mesher;

extern "C" {

int gf_mesher_create(int32_t nx, int32_t ny, int32_t nz, float dx, void *cuda_stream,
                     void **mesher_out) {
  if (!mesher_out || nx < 1 || ny < 1 || nz < 1 || !(dx > 0.f)) return GF_INVALID_ARG;
  *mesher_out = nullptr;
  const int64_t nnode = (int64_t)nx * ny * nz;
  if (nnode > (int64_t)1 << 31) return GF_INVALID_ARG;
  Mesher *m = new Mesher();
  m->nx = nx;
  m->ny = ny;
  m->nz = nz;
  m->dx = dx;
  m->nnode = nnode;
  m->nb = (int)((nnode + gfm::MB - 1) / gfm::MB);
  m->stream = reinterpret_cast<cudaStream_t>(cuda_stream);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&m->dens, nnode * 4);
  if (e == cudaSuccess) e = cudaMalloc(&m->tmp, nnode * 4);
  if (e == cudaSuccess) e = cudaMalloc(&m->vmask, nnode);
  if (e == cudaSuccess) e = cudaMalloc(&m->cmask, nnode);
  if (e == cudaSuccess) e = cudaMalloc(&m->vbase, nnode * 4);
  if (e == cudaSuccess) e = cudaMalloc(&m->sums, (4 * (int64_t)m->nb + 2) * 8);
  if (e == cudaSuccess) e = cudaMallocHost(&m->tot_host, 2 * 8);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->dens, 0, nnode * 4, m->stream);
  if (e == cudaSuccess) {  // the case table, once per device (constant memory)
    static const gfm::McTable table = gfm::build_mc_table();
    e = cudaMemcpyToSymbolAsync(gfm::c_mc, &table, sizeof(table), 0, cudaMemcpyHostToDevice,
                                m->stream);
  }
  if (e != cudaSuccess) {
    gfm::release(m);
    delete m;
    return GF_CUDA_ERROR;
  }
  *mesher_out = m;
  return GF_OK;
}

int gf_mesher_destroy(void *mesher) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m) return GF_INVALID_ARG;
  cudaStreamSynchronize(m->stream);
  gfm::release(m);
  delete m;
  return GF_OK;
}

const char *gf_mesher_last_error(void *mesher) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  return m ? m->err.c_str() : "null mesher";
}

int gf_mesher_set_stream(void *mesher, void *cuda_stream) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m) return GF_INVALID_ARG;
  m->stream = reinterpret_cast<cudaStream_t>(cuda_stream);
  return GF_OK;
}

float *gf_mesher_field(void *mesher) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  return m ? m->dens : nullptr;
}

int gf_mesher_copy_field(void *mesher, float *out) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m || !out) return GF_INVALID_ARG;
  int e = gfm::check(m, cudaMemcpyAsync(out, m->dens, m->nnode * 4, cudaMemcpyDefault, m->stream),
                     "copy mesh field");
  if (e) return e;
  return gfm::check(m, cudaStreamSynchronize(m->stream), "mesh field sync");
}

int64_t gf_mesher_launches(void *mesher) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  return m ? m->launches : -1;
}

int gf_mesher_density(void *mesher, const float *pos, int64_t n,
                      const gf_mesh_params *prm) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m || !prm || n < 0 || (n > 0 && !pos)) return GF_INVALID_ARG;
  if (prm->smooth_passes < 0 || prm->wall_margin_cells < 0)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_density: negative pass count or margin");
  if (prm->method != GF_MESH_TRILINEAR && prm->method != GF_MESH_CUBIC &&
      prm->method != GF_MESH_SDF)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_density: unknown mesh method");
  if (prm->method == GF_MESH_CUBIC && !(prm->cubic_radius_cells > 0.f))
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_density: cubic radius must be > 0");
  if (prm->method == GF_MESH_SDF &&
      !(prm->sdf_search_radius_cells > 0.f && prm->sdf_particle_radius_cells >= 0.f))
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_density: bad sdf radii");
  cudaStream_t st = m->stream;
  const unsigned gc = (unsigned)((m->nnode + 255) / 256);
  if (prm->method == GF_MESH_SDF) {
    // surface.py:405-420: radii in cells times dx (double), passed as float;
    // no wall margin (a zeroed wall would be a false surface)
    const float R = (float)((double)prm->sdf_search_radius_cells * (double)m->dx);
    const float r = (float)((double)prm->sdf_particle_radius_cells * (double)m->dx);
    const float r2 = R * R;
    unsigned *bits = reinterpret_cast<unsigned *>(m->dens);
    gfm::k_sdf_init<<<gc, 256, 0, st>>>(bits, m->nnode, r2);
    if (n > 0)
      gfm::k_sdf_scatter<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
          pos, n, m->dx, R, r2, m->nx, m->ny, m->nz, bits);
    gfm::k_sdf_finish<<<gc, 256, 0, st>>>(m->dens, m->nnode, r);
    m->launches += n > 0 ? 3 : 2;
    for (int p = 0; p < prm->smooth_passes; ++p) {
      gfm::k_mesh_blur<<<gc, 256, 0, st>>>(m->dens, m->tmp, m->nx, m->ny, m->nz, 0);
      float *t = m->dens;
      m->dens = m->tmp;
      m->tmp = t;
      m->launches++;
    }
    m->below = 1;
    m->nv = m->nt = -1;
    return gfm::check(m, cudaGetLastError(), "gf_mesher_density");
  }
  m->below = 0;
  gfm::k_mesh_zero<<<gc, 256, 0, st>>>(m->dens, m->nnode);
  m->launches++;
  if (n > 0) {
    const unsigned gp = (unsigned)((n + 255) / 256);
    if (prm->method == GF_MESH_TRILINEAR) {
      gfm::k_mesh_splat<<<gp, 256, 0, st>>>(pos, n, m->dx, m->nx, m->ny, m->nz, m->dens);
    } else {
      // surface.py:376-382: radius and falloff scale in double, passed as float
      const double r_world = (double)prm->cubic_radius_cells * (double)m->dx;
      const float inv_r_world_sq = (float)(1.0 / (r_world * r_world));
      const int half_cells = (int)std::ceil((double)prm->cubic_radius_cells) + 1;
      gfm::k_mesh_cubic<<<gp, 256, 0, st>>>(pos, n, m->dx, inv_r_world_sq, half_cells, m->nx,
                                            m->ny, m->nz, m->dens);
    }
    m->launches++;
  }
  for (int p = 0; p < prm->smooth_passes; ++p) {
    const int margin = p == prm->smooth_passes - 1 ? prm->wall_margin_cells : 0;
    gfm::k_mesh_blur<<<gc, 256, 0, st>>>(m->dens, m->tmp, m->nx, m->ny, m->nz, margin);
    float *t = m->dens;
    m->dens = m->tmp;
    m->tmp = t;
    m->launches++;
  }
  if (prm->smooth_passes == 0 && prm->wall_margin_cells > 0) {
    gfm::k_mesh_walls<<<gc, 256, 0, st>>>(m->dens, m->nx, m->ny, m->nz, prm->wall_margin_cells);
    m->launches++;
  }
  m->nv = m->nt = -1;
  return gfm::check(m, cudaGetLastError(), "gf_mesher_density");
}

int gf_mesher_extract(void *mesher, const float *field, float iso_level, int64_t *n_verts,
                      int64_t *n_tris) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m || !n_verts || !n_tris || !std::isfinite(iso_level)) return GF_INVALID_ARG;
  if (m->nx < 2 || m->ny < 2 || m->nz < 2) {  // no cube: no surface
    m->nv = m->nt = 0;
    *n_verts = *n_tris = 0;
    return GF_OK;
  }
  cudaStream_t st = m->stream;
  gfm::ExtractArgs a{field ? field : m->dens, iso_level, m->below,
                     m->surface == GF_SURFACE_MARCHING_CUBES ? 1 : 0, m->nx, m->ny, m->nz,
                     m->nnode, m->dx,
                     m->vmask, m->cmask, m->vbase, m->sums, m->nb, nullptr, nullptr};
  gfm::k_mesh_count<<<m->nb, gfm::MB, 0, st>>>(a);
  gfm::k_mesh_scan<<<2, gfm::SCAN_T, 0, st>>>(m->sums, m->nb);
  m->launches += 2;
  int e;
  if ((e = gfm::check(m, cudaGetLastError(), "gf_mesher_extract count"))) return e;
  if ((e = gfm::check(m, cudaMemcpyAsync(m->tot_host, m->sums + 4 * (int64_t)m->nb, 16,
                                         cudaMemcpyDeviceToHost, st),
                      "read mesh totals")))
    return e;
  if ((e = gfm::check(m, cudaStreamSynchronize(st), "mesh totals sync"))) return e;
  const int64_t nv = m->tot_host[0], nt = m->tot_host[1];
  if (nv > INT32_MAX)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_extract: vertex count exceeds int32 range");
  if ((e = gfm::grow(m, reinterpret_cast<void **>(&m->verts), &m->verts_cap, nv, 12,
                     "alloc mesh vertices")))
    return e;
  if ((e = gfm::grow(m, reinterpret_cast<void **>(&m->tris), &m->tris_cap, nt, 12,
                     "alloc mesh triangles")))
    return e;
  a.verts = m->verts;
  a.tris = m->tris;
  if (nv > 0) {
    gfm::k_mesh_vemit<<<m->nb, gfm::MB, 0, st>>>(a);
    gfm::k_mesh_temit<<<m->nb, gfm::MB, 0, st>>>(a);
    m->launches += 2;
  }
  m->nv = nv;
  m->nt = nt;
  *n_verts = nv;
  *n_tris = nt;
  return gfm::check(m, cudaGetLastError(), "gf_mesher_extract emit");
}

int gf_marching_cubes_table(uint8_t *edges, uint8_t *ntri, uint8_t *tri) {
  if (!edges || !ntri || !tri) return GF_INVALID_ARG;
  static const gfm::McTable table = gfm::build_mc_table();
  memcpy(edges, table.edge, sizeof(table.edge));
  memcpy(ntri, table.ntri, sizeof(table.ntri));
  memcpy(tri, table.tri, sizeof(table.tri));
  return GF_OK;
}

int gf_mesher_set_surface(void *mesher, int32_t method) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m) return GF_INVALID_ARG;
  if (method != GF_SURFACE_MARCHING_CUBES && method != GF_SURFACE_MARCHING_TETRAHEDRA)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_set_surface: unknown method");
  m->surface = method;
  return GF_OK;
}

int gf_mesher_set_inside_below(void *mesher, int32_t below) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m) return GF_INVALID_ARG;
  m->below = below ? 1 : 0;
  return GF_OK;
}

int gf_mesher_copy(void *mesher, float *verts, int32_t *tris) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m) return GF_INVALID_ARG;
  if (m->nv < 0) return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_copy: no extraction to copy");
  if ((m->nv > 0 && !verts) || (m->nt > 0 && !tris)) return GF_INVALID_ARG;
  int e;
  if (m->nv > 0 &&
      (e = gfm::check(m, cudaMemcpyAsync(verts, m->verts, m->nv * 12, cudaMemcpyDefault,
                                         m->stream),
                      "copy mesh vertices")))
    return e;
  if (m->nt > 0 &&
      (e = gfm::check(m, cudaMemcpyAsync(tris, m->tris, m->nt * 12, cudaMemcpyDefault,
                                         m->stream),
                      "copy mesh triangles")))
    return e;
  return gfm::check(m, cudaStreamSynchronize(m->stream), "mesh copy sync");
}

int gf_mesher_smooth(void *mesher, float *verts, int64_t n_verts, const int32_t *tris,
                     int64_t n_tris, int32_t method, int32_t passes, double lam, double mu) {
  Mesher *m = reinterpret_cast<Mesher *>(mesher);
  if (!m || passes < 0 || n_verts < 0 || n_tris < 0) return GF_INVALID_ARG;
  if (method != GF_MESH_SMOOTH_LAPLACIAN && method != GF_MESH_SMOOTH_TAUBIN)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_smooth: unknown smoothing method");
  if (!verts) {  // the last extraction
    if (m->nv < 0) return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_smooth: no extraction");
    verts = m->verts;
    n_verts = m->nv;
    tris = m->tris;
    n_tris = m->nt;
  } else if (n_tris > 0 && !tris) {
    return GF_INVALID_ARG;
  }
  if (n_verts > INT32_MAX || 6 * n_tris > INT32_MAX)
    return gfm::fail(m, GF_INVALID_ARG, "gf_mesher_smooth: mesh exceeds int32 indexing");
  if (passes == 0 || n_verts == 0) return GF_OK;
  return gfm::smooth(m, verts, n_verts, tris, n_tris, method, passes, lam, mu);
}

}  // extern "C"
