// Particle <-> grid transfers and the explicit grid stages of one substep.
//
//   k_p2g_tile<APIC>  k3_p2g (solver3d.py:72-114) / k3_p2g_apic (:1475-1588):
//                     one CTA per 8x8x8 cell tile; the tile's sorted particles
//                     scatter into a shared-memory box covering every face
//                     they can touch; the box is flushed with plain stores on
//                     faces no other tile reaches and float atomics on the
//                     one-cell halo band shared with neighbouring tiles.
//   k_forces          k3_normalize (:121-142) + k3_add_gravity (:149-156) +
//                     k3_enforce_solid_bc (:758-799) in one pass over faces.
//   k_divergence      k3_compute_divergence (:846-871).
//   k_project         k3_subtract_pressure_grad (:1364-1407) + the second
//                     k3_enforce_solid_bc of _step_impl (:3635-3642).
//   k_g2p<MODE>       k3_g2p_and_advect (:1414-1463) / k3_g2p_apic_advect
//                     (:1591-1732) over sorted particles; results go back to
//                     the caller's AoS buffers in sorted order (pid follows).
//
// This unit is compiled with -fmad=false: every product and sum rounds
// separately, in the reference's operation order, so that each stage is
// bit-identical to the CPU oracle when its inputs are.  Only the order of the
// floating-point atomic sums in P2G differs (P2G uses explicit fused
// multiply-adds, its sums being tolerance-checked).  G2P does part of its
// arithmetic on packed float32 pairs (mul2 / sum2 of gf_internal.cuh), each
// half rounded as the scalar operation, so it stays bit-identical.
#include "gf_internal.cuh"

namespace gf {

// ---------------------------------------------------------------- P2G
// A CTA scatters a block of KT tiles along k (8 x 8 x 8 KT cells; KT = 1 or
// 2, chosen by the autotuner) into shared-memory boxes, in faces, relative to
// the block origin (I0, J0, K0): on the i and j axes the normal axis spans
// [O, O+8] (9 faces) and the transverse ones [O-1, O+8] (10 faces); on the k
// axis [K0, K0+8KT] for w and [K0-1, K0+8KT] for u and v.  Each component's
// box takes P2G_BOXK(KT) entries (the largest of the three).
constexpr int BOX_N = 9, BOX_T = 10;
__host__ __device__ constexpr int p2g_ez(int comp, int KT) {
  return comp == 2 ? 8 * KT + 1 : 8 * KT + 2;
}
__host__ __device__ constexpr int P2G_BOXK(int KT) { return BOX_T * BOX_T * (8 * KT + 1); }
static_assert(P2G_BOXK(1) == 900 && BOX_N * BOX_T * 10 <= P2G_BOXK(1), "P2G box");
// Type of the shared-memory face sums of a tile (the sums are rounded to
// float32 once, at the flush).
#ifndef GF_P2G_ACC
#define GF_P2G_ACC float
#endif
using P2G_ACC = GF_P2G_ACC;

struct P2GArgs {
  const int32_t *start;
  const float4 *rec0, *rec1, *rec2, *rec3;
  float *u, *v, *w, *uw, *vw, *ww;
  float dx;
  int nx, ny, nz, nty, ntz;
  float inv_dx_exact;  // exact_inverse(dx)
};


// Scatter one face component of one particle into the shared box of `comp`
// (0 u, 1 v, 2 w).  APIC adds C_row . (x_face - x_p) with world face
// positions (:1510-1588).
template <bool APIC, int KT, typename T>
__device__ __forceinline__ void scatter_comp(T *s_val, T *s_wt, int comp, float vp,
                                             float c0, float c1, float c2, float px, float py,
                                             float pz, float fx, float fy, float fz, int I0,
                                             int J0, int K0, const P2GArgs &a, float *gval,
                                             float *gwt) {
  int snx = a.nx + (comp == 0), sny = a.ny + (comp == 1), snz = a.nz + (comp == 2);
  int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
      k0 = __float2int_rz(floorf(fz));
  float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  // box origin and extents for this component
  int bx0 = comp == 0 ? I0 : I0 - 1, by0 = comp == 1 ? J0 : J0 - 1, bz0 = comp == 2 ? K0 : K0 - 1;
  int ey = comp == 1 ? BOX_N : BOX_T, ez = p2g_ez(comp, KT);
  int ex = comp == 0 ? BOX_N : BOX_T;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        int ii = i0 + di, jj = j0 + dj, kk = k0 + dk;
        if (ii >= 0 && ii < snx && jj >= 0 && jj < sny && kk >= 0 && kk < snz) {
          float wxi = di == 0 ? 1.0f - sx : sx;
          float wyi = dj == 0 ? 1.0f - sy : sy;
          float wzi = dk == 0 ? 1.0f - sz : sz;
          float wt = wxi * wyi;
          wt = wt * wzi;
          float val = vp;
          if (APIC) {
            float ox = comp == 0 ? (float)ii * a.dx - px : ((float)ii + 0.5f) * a.dx - px;
            float oy = comp == 1 ? (float)jj * a.dx - py : ((float)jj + 0.5f) * a.dx - py;
            float oz = comp == 2 ? (float)kk * a.dx - pz : ((float)kk + 0.5f) * a.dx - pz;
            float t0 = c0 * ox, t1 = c1 * oy, t2 = c2 * oz;
            val = vp + t0;
            val = val + t1;
            val = val + t2;
          }
          float add = val * wt;
          int bx = ii - bx0, by = jj - by0, bz = kk - bz0;
          if (bx >= 0 && bx < ex && by >= 0 && by < ey && bz >= 0 && bz < ez) {
            int e = (bx * ey + by) * ez + bz;
            atomicAdd(&s_val[e], (T)add);
            atomicAdd(&s_wt[e], (T)wt);
          } else {  // only reachable for positions outside their clamped cell
            int64_t g = ((int64_t)ii * sny + jj) * snz + kk;
            if (GF_IN(g, (int64_t)snx * sny * snz)) {
              atomicAdd(&gval[g], add);
              atomicAdd(&gwt[g], wt);
            }
          }
        }
      }
}

// The common case of scatter_comp: the particle's 2x2x2 stencil lies inside
// the grid and inside the tile's box, so no corner needs a bounds check.  The
// per-axis factors are formed once -- weights (1-s, s), and for APIC the
// affine terms vp + c0 ox, c1 oy, c2 oz at both corners of each axis (ox one
// dx apart) -- and each corner costs two products, two adds and the two
// shared-memory adds.  The sums are tolerance-checked (their order is the
// atomics' anyway), so the factors use fused multiply-adds.  Returns false,
// touching nothing, when the stencil does not fit (scatter_comp then runs).
template <bool APIC, int KT, typename T>
__device__ __forceinline__ bool scatter_comp_fast(T *s_val, T *s_wt, int comp, float vp,
                                                  float c0, float c1, float c2, float px,
                                                  float py, float pz, float fx, float fy,
                                                  float fz, int I0, int J0, int K0,
                                                  const P2GArgs &a) {
  const int snx = a.nx + (comp == 0), sny = a.ny + (comp == 1), snz = a.nz + (comp == 2);
  const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
            k0 = __float2int_rz(floorf(fz));
  const int ey = comp == 1 ? BOX_N : BOX_T, ez = p2g_ez(comp, KT);
  const int ex = comp == 0 ? BOX_N : BOX_T;
  const int bx = i0 - (comp == 0 ? I0 : I0 - 1), by = j0 - (comp == 1 ? J0 : J0 - 1),
            bz = k0 - (comp == 2 ? K0 : K0 - 1);
  if (!(i0 >= 0 && i0 + 1 < snx && j0 >= 0 && j0 + 1 < sny && k0 >= 0 && k0 + 1 < snz &&
        bx >= 0 && bx + 1 < ex && by >= 0 && by + 1 < ey && bz >= 0 && bz + 1 < ez))
    return false;
  const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
  float A[2] = {vp, vp}, B[2] = {0.f, 0.f}, C[2] = {0.f, 0.f};
  if (APIC) {
    const float dx = a.dx;
    const float ox = ((float)i0 + (comp == 0 ? 0.0f : 0.5f)) * dx - px;
    const float oy = ((float)j0 + (comp == 1 ? 0.0f : 0.5f)) * dx - py;
    const float oz = ((float)k0 + (comp == 2 ? 0.0f : 0.5f)) * dx - pz;
    A[0] = __fmaf_rn(c0, ox, vp);
    A[1] = __fmaf_rn(c0, dx, A[0]);
    B[0] = c1 * oy;
    B[1] = __fmaf_rn(c1, dx, B[0]);
    C[0] = c2 * oz;
    C[1] = __fmaf_rn(c2, dx, C[0]);
  }
  const int base = (bx * ey + by) * ez + bz;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const float wxy = wx[di] * wy[dj];
      const float ab = A[di] + B[dj];
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const float wt = wxy * wz[dk];
        const float val = ab + C[dk];
        const int e = base + (di * ey + dj) * ez + dk;
        if (!GF_IN(e, P2G_BOXK(KT))) continue;
        atomicAdd(&s_val[e], (T)(val * wt));
        atomicAdd(&s_wt[e], (T)wt);
      }
    }
  return true;
}

// Flush a tile's shared box: faces that only this tile's particles reach are
// stored, the shared halo band is accumulated atomically; exact zeros are
// skipped (the destination was zeroed before the launch).  One component at
// a time, so the box extents are compile-time constants and the entry index
// splits into (bx, by, bz) by multiplications instead of divisions.
template <int COMP, int KT, typename T>
__device__ __forceinline__ void p2g_flush_comp(const P2GArgs &a, const T *s_val, const T *s_wt,
                                               int I0, int J0, int K0) {
  constexpr int EX = COMP == 0 ? BOX_N : BOX_T, EY = COMP == 1 ? BOX_N : BOX_T,
                EZ = p2g_ez(COMP, KT);
  const int snx = a.nx + (COMP == 0), sny = a.ny + (COMP == 1), snz = a.nz + (COMP == 2);
  const int ox = COMP == 0 ? I0 : I0 - 1, oy = COMP == 1 ? J0 : J0 - 1,
            oz = COMP == 2 ? K0 : K0 - 1;
  float *const gv = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
  float *const gw = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);
  for (int e2 = threadIdx.x; e2 < EX * EY * EZ; e2 += blockDim.x) {
    const float val = (float)s_val[e2], wt = (float)s_wt[e2];
    if (val == 0.f && wt == 0.f) continue;
    const int bx = e2 / (EY * EZ), by = (e2 / EZ) % EY, bz = e2 % EZ;
    const int ii = bx + ox, jj = by + oy, kk = bz + oz;
    if (ii < 0 || ii >= snx || jj < 0 || jj >= sny || kk < 0 || kk >= snz) continue;
    // exclusive: every cell that can reach the face lies in this tile
    const bool ex_x = COMP == 0 ? (bx >= 1 && bx <= 7) : (bx >= 2 && bx <= 7);
    const bool ex_y = COMP == 1 ? (by >= 1 && by <= 7) : (by >= 2 && by <= 7);
    const bool ex_z = COMP == 2 ? (bz >= 1 && bz <= 8 * KT - 1) : (bz >= 2 && bz <= 8 * KT - 1);
    const int64_t g = ((int64_t)ii * sny + jj) * snz + kk;
    if (!GF_IN(g, (int64_t)snx * sny * snz)) continue;
    if (ex_x && ex_y && ex_z) {
      gv[g] = val;
      gw[g] = wt;
    } else {
      atomicAdd(&gv[g], val);
      atomicAdd(&gw[g], wt);
    }
  }
}

template <int KT, typename T>
__device__ __forceinline__ void p2g_flush_box(const P2GArgs &a, const T *s_val, const T *s_wt,
                                              int I0, int J0, int K0) {
  constexpr int BK = P2G_BOXK(KT);
  p2g_flush_comp<0, KT, T>(a, s_val, s_wt, I0, J0, K0);
  p2g_flush_comp<1, KT, T>(a, s_val + BK, s_wt + BK, I0, J0, K0);
  p2g_flush_comp<2, KT, T>(a, s_val + 2 * BK, s_wt + 2 * BK, I0, J0, K0);
}

// Per-cell register accumulation (p2g_map 2), one face component COMP: lane
// l owns cell (ci, cj, ck) and sums the contributions of all its particles
// to the union of their stencils -- 2 faces along the component's normal
// axis (i0 = the cell index), 3 along each transverse one (i0 = cell - 1 or
// cell) -- in 18 register pairs, then adds the non-empty sums to the box: at
// most 36 shared atomics per cell and component where scattering particle by
// particle costs 16 per particle.  At each step of the flush the lanes add to
// distinct faces (distinct cells, one common offset).  Each corner weight is
// wx * wy * wz with zero factors off the particle's own 2 x 2 x 2 corners,
// so the per-face sums are those of the particle-by-particle scatter in
// another order.  A particle whose stencil does not start in its cell's
// pattern (a position outside the grid, binned into a boundary cell) goes
// through scatter_comp.
template <bool APIC, int KT, int COMP, typename T>
__device__ __forceinline__ void p2g_cell_comp(const P2GArgs &a, T *s_val, T *s_wt, int64_t first,
                                              int cnt, int maxcnt, int ci, int cj, int ck,
                                              int I0, int J0, int K0) {
  constexpr int EX = COMP == 0 ? 2 : 3, EY = COMP == 1 ? 2 : 3, EZ = COMP == 2 ? 2 : 3;
  constexpr float HX = COMP == 0 ? 0.0f : 0.5f, HY = COMP == 1 ? 0.0f : 0.5f,
                  HZ = COMP == 2 ? 0.0f : 0.5f;
  const int xo = ci - (COMP != 0), yo = cj - (COMP != 1), zo = ck - (COMP != 2);
  const float dx = a.dx, inv = a.inv_dx_exact;
  // (value, weight) sums of each face, one f32x2 pair
  float2 acc[EX * EY * EZ];
#pragma unroll
  for (int m = 0; m < EX * EY * EZ; ++m) acc[m] = dup2(0.0f);
  for (int kp = 0; kp < maxcnt; ++kp) {
    if (kp >= cnt) continue;
    const int64_t q = first + kp;
    const float4 r0 = a.rec0[q];
    float vp, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    // APIC: record 1 + c holds (v_c, C row c); FLIP/PIC: record 1 (vx, vy, vz)
    if (APIC) {
      const float4 rc = (COMP == 0 ? a.rec1 : (COMP == 1 ? a.rec2 : a.rec3))[q];
      vp = rc.x; c0 = rc.y; c1 = rc.z; c2 = rc.w;
    } else {
      const float4 r1 = a.rec1[q];
      vp = COMP == 0 ? r1.x : (COMP == 1 ? r1.y : r1.z);
    }
    // x / dx: a product when dx is a power of two (exact), else the division
    const float gx = div_dx(r0.x, dx, inv);
    const float gy = div_dx(r0.y, dx, inv);
    const float gz = div_dx(r0.z, dx, inv);
    const float fx = gx - HX, fy = gy - HY, fz = gz - HZ;
    const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
              k0 = __float2int_rz(floorf(fz));
    const int rx = i0 - xo, ry = j0 - yo, rz = k0 - zo;
    if (rx < 0 || rx + 2 > EX || ry < 0 || ry + 2 > EY || rz < 0 || rz + 2 > EZ) {
      float *gv = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
      float *gw = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);
      scatter_comp<APIC, KT, T>(s_val, s_wt, COMP, vp, c0, c1, c2, r0.x, r0.y, r0.z, fx, fy, fz,
                                I0, J0, K0, a, gv, gw);
      continue;
    }
    const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
    float wx[EX], wy[EY], wz[EZ], A[EX], B[EY], C[EZ];
#pragma unroll
    for (int m = 0; m < EX; ++m) {
      wx[m] = m == rx ? 1.0f - sx : (m == rx + 1 ? sx : 0.0f);
      A[m] = APIC ? __fmaf_rn(c0, ((float)(xo + m) + HX) * dx - r0.x, vp) : vp;
    }
#pragma unroll
    for (int m = 0; m < EY; ++m) {
      wy[m] = m == ry ? 1.0f - sy : (m == ry + 1 ? sy : 0.0f);
      B[m] = APIC ? c1 * (((float)(yo + m) + HY) * dx - r0.y) : 0.0f;
    }
#pragma unroll
    for (int m = 0; m < EZ; ++m) {
      wz[m] = m == rz ? 1.0f - sz : (m == rz + 1 ? sz : 0.0f);
      C[m] = APIC ? c2 * (((float)(zo + m) + HZ) * dx - r0.z) : 0.0f;
    }
    // face (x, y, z) gains (A_x + B_y + C_z) wx wy wz, summed as
    // (wxy (A_x + B_y)) wz + wxy (C_z wz) with wxy = wx wy, and weight wxy wz
    float D[EZ];
#pragma unroll
    for (int z = 0; z < EZ; ++z) D[z] = C[z] * wz[z];
#pragma unroll
    for (int x = 0; x < EX; ++x)
#pragma unroll
      for (int y = 0; y < EY; ++y) {
        const float wxy = wx[x] * wy[y];
        const float P = wxy * (A[x] + B[y]);
#pragma unroll
        for (int z = 0; z < EZ; ++z) {
          const int m = (x * EY + y) * EZ + z;
          acc[m] = fma2(make_float2(P, wxy), dup2(wz[z]), acc[m]);
          if (APIC) acc[m].x = __fmaf_rn(wxy, D[z], acc[m].x);
        }
      }
  }
  // box offsets: the register origin (xo, yo, zo) sits at box entry
  // (ci - I0, cj - J0, ck - K0) of this component's box
  const int ey = COMP == 1 ? BOX_N : BOX_T, ez = p2g_ez(COMP, KT);
  const int e0 = ((ci - I0) * ey + (cj - J0)) * ez + (ck - K0);
#pragma unroll
  for (int x = 0; x < EX; ++x)
#pragma unroll
    for (int y = 0; y < EY; ++y)
#pragma unroll
      for (int z = 0; z < EZ; ++z) {
        const int m = (x * EY + y) * EZ + z;
        if (acc[m].y == 0.0f) continue;
        const int e = e0 + (x * ey + y) * ez + z;
        if (!GF_IN(e, P2G_BOXK(KT))) continue;
        atomicAdd(&s_val[e], (T)acc[m].x);
        atomicAdd(&s_wt[e], (T)acc[m].y);
      }
}

// Lane map 3: the cells of map 2, with the particles read from a warp-private
// shared staging area instead of global memory.  A warp's 32 cells hold one
// contiguous range of the sorted particles; it is loaded P2G_CH particles at
// a time with coalesced 16-byte loads (lane i takes particles i, i + 32, ...)
// into structure-of-arrays fields -- grid coordinates x/dx, velocity, and for
// APIC the world position and the 3 x 3 C -- and each lane then sums its own
// cell's particles of the chunk from there.  Reading a cell's particles
// straight from global memory (map 2) makes every load instruction touch 32
// different cache lines.
constexpr int P2G_CH = 128;  // particles per warp and chunk
__host__ __device__ constexpr int p2g_stage_fields(bool apic) { return apic ? 18 : 6; }
// field f of staged particle i: s[f * P2G_CH + i]
//   0..2 x/dx, y/dx, z/dx   3..5 vx, vy, vz   (APIC) 6..8 x, y, z   9..17 C row-major
template <bool APIC, int KT, int COMP, typename T>
__device__ __forceinline__ void p2g_cell_comp_staged(const P2GArgs &a, T *s_val, T *s_wt,
                                                     const float *st, int lo, int cnt,
                                                     int maxcnt, int ci, int cj, int ck, int I0,
                                                     int J0, int K0) {
  constexpr int EX = COMP == 0 ? 2 : 3, EY = COMP == 1 ? 2 : 3, EZ = COMP == 2 ? 2 : 3;
  constexpr float HX = COMP == 0 ? 0.0f : 0.5f, HY = COMP == 1 ? 0.0f : 0.5f,
                  HZ = COMP == 2 ? 0.0f : 0.5f;
  const int xo = ci - (COMP != 0), yo = cj - (COMP != 1), zo = ck - (COMP != 2);
  const float dx = a.dx;
  float av[EX * EY * EZ], aw[EX * EY * EZ];
#pragma unroll
  for (int m = 0; m < EX * EY * EZ; ++m) av[m] = aw[m] = 0.0f;
  for (int kp = 0; kp < maxcnt; ++kp) {
    if (kp >= cnt) continue;
    const int i = lo + kp;
    const float fx = st[0 * P2G_CH + i] - HX, fy = st[1 * P2G_CH + i] - HY,
                fz = st[2 * P2G_CH + i] - HZ;
    const float vp = st[(3 + COMP) * P2G_CH + i];
    float px = 0.f, py = 0.f, pz = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    if (APIC) {
      px = st[6 * P2G_CH + i];
      py = st[7 * P2G_CH + i];
      pz = st[8 * P2G_CH + i];
      c0 = st[(9 + 3 * COMP) * P2G_CH + i];
      c1 = st[(10 + 3 * COMP) * P2G_CH + i];
      c2 = st[(11 + 3 * COMP) * P2G_CH + i];
    }
    const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
              k0 = __float2int_rz(floorf(fz));
    const int rx = i0 - xo, ry = j0 - yo, rz = k0 - zo;
    if (rx < 0 || rx + 2 > EX || ry < 0 || ry + 2 > EY || rz < 0 || rz + 2 > EZ) {
      float *gv = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
      float *gw = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);
      scatter_comp<APIC, KT, T>(s_val, s_wt, COMP, vp, c0, c1, c2, px, py, pz, fx, fy, fz, I0,
                                J0, K0, a, gv, gw);
      continue;
    }
    const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
    float wx[EX], wy[EY], wz[EZ], A[EX], B[EY], C[EZ];
#pragma unroll
    for (int m = 0; m < EX; ++m) {
      wx[m] = m == rx ? 1.0f - sx : (m == rx + 1 ? sx : 0.0f);
      A[m] = APIC ? __fmaf_rn(c0, ((float)(xo + m) + HX) * dx - px, vp) : vp;
    }
#pragma unroll
    for (int m = 0; m < EY; ++m) {
      wy[m] = m == ry ? 1.0f - sy : (m == ry + 1 ? sy : 0.0f);
      B[m] = APIC ? c1 * (((float)(yo + m) + HY) * dx - py) : 0.0f;
    }
#pragma unroll
    for (int m = 0; m < EZ; ++m) {
      wz[m] = m == rz ? 1.0f - sz : (m == rz + 1 ? sz : 0.0f);
      C[m] = APIC ? c2 * (((float)(zo + m) + HZ) * dx - pz) : 0.0f;
    }
#pragma unroll
    for (int x = 0; x < EX; ++x)
#pragma unroll
      for (int y = 0; y < EY; ++y) {
        const float wxy = wx[x] * wy[y];
        const float ab = A[x] + B[y];
#pragma unroll
        for (int z = 0; z < EZ; ++z) {
          const int m = (x * EY + y) * EZ + z;
          const float wt = wxy * wz[z];
          av[m] = __fmaf_rn(ab + C[z], wt, av[m]);
          aw[m] += wt;
        }
      }
  }
  const int ey = COMP == 1 ? BOX_N : BOX_T, ez = p2g_ez(COMP, KT);
  const int e0 = ((ci - I0) * ey + (cj - J0)) * ez + (ck - K0);
#pragma unroll
  for (int x = 0; x < EX; ++x)
#pragma unroll
    for (int y = 0; y < EY; ++y)
#pragma unroll
      for (int z = 0; z < EZ; ++z) {
        const int m = (x * EY + y) * EZ + z;
        if (aw[m] == 0.0f) continue;
        const int e = e0 + (x * ey + y) * ez + z;
        if (!GF_IN(e, P2G_BOXK(KT))) continue;
        atomicAdd(&s_val[e], (T)av[m]);
        atomicAdd(&s_wt[e], (T)aw[m]);
      }
}

// Lane maps 4 and 5: the cells of map 2, with the particles staged in
// rounds of up to K (8 or 4) per cell by the whole warp.  In a round, slot s
// of cell l holds the cell's (K r + s)-th particle; the warp loads the slots
// in K steps of 32 / K cells, lane j of step t taking slot j % K of cell
// (32 / K) t + j / K, so a load instruction reads 32 / K runs of K
// consecutive sorted particles.  Slot s of cell l lives at s * 32 + (l ^
// (32 / K) s) of each field's plane: a step's stores and a lane's reads of its
// own cell (all lanes at one slot) both fall in 32 distinct banks.  One face
// component at a time (its register sums live across the rounds), each
// staged field being one of: the grid coordinates x/dx, y/dx, z/dx (unshifted),
// v_c, and for APIC the row c of C.  The APIC offsets are formed in grid units,
// (face - x/dx) dx, so the world position is not staged.
template <bool APIC>
__host__ __device__ constexpr int p2g_round_fields() { return APIC ? 7 : 4; }
template <int K>
__device__ __forceinline__ int p2g_round_slot(int cell, int s) {
  return s * 32 + (cell ^ ((32 / K) * s));
}
template <bool APIC, int KT, int COMP, int K, typename T>
__device__ __forceinline__ void p2g_cell_comp_rounds(const P2GArgs &a, T *s_val, T *s_wt,
                                                     float *st, int64_t first, int cnt,
                                                     int maxcnt, int ci, int cj, int ck, int I0,
                                                     int J0, int K0) {
  constexpr int EX = COMP == 0 ? 2 : 3, EY = COMP == 1 ? 2 : 3, EZ = COMP == 2 ? 2 : 3;
  constexpr float HX = COMP == 0 ? 0.0f : 0.5f, HY = COMP == 1 ? 0.0f : 0.5f,
                  HZ = COMP == 2 ? 0.0f : 0.5f;
  constexpr int PL = K * 32;  // slots of a field's plane
  const int lane = threadIdx.x & 31;
  const int xo = ci - (COMP != 0), yo = cj - (COMP != 1), zo = ck - (COMP != 2);
  const float dx = a.dx, inv = a.inv_dx_exact;
  const float4 *recc = APIC ? (COMP == 0 ? a.rec1 : (COMP == 1 ? a.rec2 : a.rec3)) : a.rec1;
  float av[EX * EY * EZ], aw[EX * EY * EZ];
#pragma unroll
  for (int m = 0; m < EX * EY * EZ; ++m) av[m] = aw[m] = 0.0f;
  for (int kb = 0; kb < maxcnt; kb += K) {
    __syncwarp();
    // ---- stage the round: K steps of 32 / K cells
#pragma unroll
    for (int t = 0; t < K; ++t) {
      const int cc = (32 / K) * t + lane / K, s = lane % K;
      const int64_t fc = __shfl_sync(0xffffffffu, first, cc);
      const int nc = __shfl_sync(0xffffffffu, cnt, cc);
      if (kb + s < nc) {
        const int64_t q = fc + kb + s;
        const float4 r0 = a.rec0[q], rc = recc[q];
        const int o = p2g_round_slot<K>(cc, s);
        st[0 * PL + o] = div_dx(r0.x, dx, inv);
        st[1 * PL + o] = div_dx(r0.y, dx, inv);
        st[2 * PL + o] = div_dx(r0.z, dx, inv);
        if (APIC) {  // record 1 + c: (v_c, C row c)
          st[3 * PL + o] = rc.x;
          st[4 * PL + o] = rc.y;
          st[5 * PL + o] = rc.z;
          st[6 * PL + o] = rc.w;
        } else {
          st[3 * PL + o] = COMP == 0 ? rc.x : (COMP == 1 ? rc.y : rc.z);
        }
      }
    }
    __syncwarp();
    // ---- this lane's cell: its particles kb .. kb + K - 1
#pragma unroll 1
    for (int s = 0; s < K; ++s) {
      if (kb + s >= cnt) break;
      const int o = p2g_round_slot<K>(lane, s);
      const float gx = st[0 * PL + o], gy = st[1 * PL + o], gz = st[2 * PL + o];
      const float fx = gx - HX, fy = gy - HY, fz = gz - HZ;
      const float vp = st[3 * PL + o];
      float c0 = 0.f, c1 = 0.f, c2 = 0.f;
      if (APIC) {
        c0 = st[4 * PL + o];
        c1 = st[5 * PL + o];
        c2 = st[6 * PL + o];
      }
      const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
                k0 = __float2int_rz(floorf(fz));
      const int rx = i0 - xo, ry = j0 - yo, rz = k0 - zo;
      if (rx < 0 || rx + 2 > EX || ry < 0 || ry + 2 > EY || rz < 0 || rz + 2 > EZ) {
        // outside the cell's pattern (a position outside the grid): the
        // general scatter, with the world position rebuilt from the record
        const float4 r0 = a.rec0[first + kb + s];
        float *gv = COMP == 0 ? a.u : (COMP == 1 ? a.v : a.w);
        float *gw = COMP == 0 ? a.uw : (COMP == 1 ? a.vw : a.ww);
        scatter_comp<APIC, KT, T>(s_val, s_wt, COMP, vp, c0, c1, c2, r0.x, r0.y, r0.z, fx, fy,
                                  fz, I0, J0, K0, a, gv, gw);
        continue;
      }
      const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
      float wx[EX], wy[EY], wz[EZ], A[EX], B[EY], C[EZ];
#pragma unroll
      for (int m = 0; m < EX; ++m) {
        wx[m] = m == rx ? 1.0f - sx : (m == rx + 1 ? sx : 0.0f);
        A[m] = APIC ? __fmaf_rn(c0, (((float)(xo + m) + HX) - gx) * dx, vp) : vp;
      }
#pragma unroll
      for (int m = 0; m < EY; ++m) {
        wy[m] = m == ry ? 1.0f - sy : (m == ry + 1 ? sy : 0.0f);
        B[m] = APIC ? c1 * ((((float)(yo + m) + HY) - gy) * dx) : 0.0f;
      }
#pragma unroll
      for (int m = 0; m < EZ; ++m) {
        wz[m] = m == rz ? 1.0f - sz : (m == rz + 1 ? sz : 0.0f);
        C[m] = APIC ? c2 * ((((float)(zo + m) + HZ) - gz) * dx) : 0.0f;
      }
#pragma unroll
      for (int x = 0; x < EX; ++x)
#pragma unroll
        for (int y = 0; y < EY; ++y) {
          const float wxy = wx[x] * wy[y];
          const float ab = A[x] + B[y];
#pragma unroll
          for (int z = 0; z < EZ; ++z) {
            const int m = (x * EY + y) * EZ + z;
            const float wt = wxy * wz[z];
            av[m] = __fmaf_rn(ab + C[z], wt, av[m]);
            aw[m] += wt;
          }
        }
    }
  }
  const int ey = COMP == 1 ? BOX_N : BOX_T, ez = p2g_ez(COMP, KT);
  const int e0 = ((ci - I0) * ey + (cj - J0)) * ez + (ck - K0);
#pragma unroll
  for (int x = 0; x < EX; ++x)
#pragma unroll
    for (int y = 0; y < EY; ++y)
#pragma unroll
      for (int z = 0; z < EZ; ++z) {
        const int m = (x * EY + y) * EZ + z;
        if (aw[m] == 0.0f) continue;
        const int e = e0 + (x * ey + y) * ez + z;
        if (!GF_IN(e, P2G_BOXK(KT))) continue;
        atomicAdd(&s_val[e], (T)av[m]);
        atomicAdd(&s_wt[e], (T)aw[m]);
      }
}

// One block's P2G: t is its first tile within the grid (the block's
// coordinates), key0 the sort key of that tile's first cell (t * 512 for a
// single grid), ntk (<= KT) the tiles it holds along k, which are consecutive
// in the sorted order.  The boxes live in dynamic shared memory
// (p2g_smem_bytes).
template <bool APIC, int KT, int MAP = 0, typename T = P2G_ACC>
__device__ __forceinline__ void p2g_tile_body(const P2GArgs &a, int t, int64_t key0, int ntk) {
  extern __shared__ __align__(16) unsigned char p2g_smem[];
  constexpr int BK = P2G_BOXK(KT);
  T *s_val = reinterpret_cast<T *>(p2g_smem);
  T *s_wt = s_val + 3 * BK;
  const int64_t b = a.start[key0], e = a.start[key0 + (int64_t)ntk * TILE_CELLS];
  if (b == e) return;
  // zero both boxes (contiguous, 16-byte aligned) with 16-byte stores
  static_assert((2 * 3 * BK * sizeof(T)) % 16 == 0, "P2G box size");
  for (int q = threadIdx.x; q < (int)(2 * 3 * BK * sizeof(T) / 16); q += blockDim.x)
    reinterpret_cast<uint4 *>(s_val)[q] = make_uint4(0u, 0u, 0u, 0u);
  __syncthreads();
  const int ti = t / (a.nty * a.ntz), tj = (t / a.ntz) % a.nty, tk = t % a.ntz;
  const int I0 = ti * TILE, J0 = tj * TILE, K0 = tk * TILE;
  // Lane-to-particle mapping (the autotuner's p2g_map):
  //  0: lane l of every warp walks its own contiguous run [l*run, (l+1)*run)
  //     of the block's cell-sorted particles, so the 32 lanes of one
  //     instruction sit about run/ppc cells apart and their shared atomics
  //     rarely share an address (consecutive lanes would hit one cell's 8
  //     corners), and every lane has the same work;
  //  1: a warp takes 32 cells at a time -- 4 rows of 8 along k, consecutive
  //     in the sort key -- and lane l the k-th particle of cell l in round k,
  //     so one instruction's atomics land on nearly consecutive box entries
  //     (few bank conflicts); lanes of emptier cells idle;
  //  2: the cells of 1, each lane summing its cell's particles in registers
  //     first, one component at a time (p2g_cell_comp);
  //  3: map 2 reading the particles from a warp-private staging area filled
  //     with coalesced loads (p2g_cell_comp_staged);
  //  4, 5: map 2 over rounds of 8 or 4 particles per cell, staged by the
  //     warp in bank-conflict-free slots (p2g_cell_comp_rounds).
  if (MAP == 4 || MAP == 5) {
    constexpr int K = MAP == 4 ? 8 : 4;
    const int lane4 = threadIdx.x & 31, warp4 = threadIdx.x >> 5;
    float *st = reinterpret_cast<float *>(s_wt + 3 * BK) +
                warp4 * p2g_round_fields<APIC>() * K * 32;
    for (int g4 = warp4; g4 < ntk * (TILE_CELLS / 32); g4 += blockDim.x >> 5) {
      const int cl = g4 * 32 + lane4;
      const int64_t key = key0 + cl;
      const int64_t first = a.start[key];
      const int cnt = (int)(a.start[key + 1] - first);
      const int maxcnt = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
      if (maxcnt == 0) continue;
      const int l = cl & (TILE_CELLS - 1);
      const int ci = I0 + (l >> 6), cj = J0 + ((l >> 3) & 7), ck = K0 + (cl >> 9) * TILE + (l & 7);
      p2g_cell_comp_rounds<APIC, KT, 0, K, T>(a, s_val, s_wt, st, first, cnt, maxcnt, ci, cj, ck,
                                              I0, J0, K0);
      p2g_cell_comp_rounds<APIC, KT, 1, K, T>(a, s_val + BK, s_wt + BK, st, first, cnt, maxcnt,
                                              ci, cj, ck, I0, J0, K0);
      p2g_cell_comp_rounds<APIC, KT, 2, K, T>(a, s_val + 2 * BK, s_wt + 2 * BK, st, first, cnt,
                                              maxcnt, ci, cj, ck, I0, J0, K0);
    }
    __syncthreads();
    p2g_flush_box<KT, T>(a, s_val, s_wt, I0, J0, K0);
    return;
  }
  if (MAP == 3) {
    const int lane3 = threadIdx.x & 31, warp3 = threadIdx.x >> 5;
    constexpr int NF = p2g_stage_fields(APIC);
    float *st = reinterpret_cast<float *>(s_wt + 3 * BK) + warp3 * NF * P2G_CH;
    const float dx = a.dx;
    for (int g3 = warp3; g3 < ntk * (TILE_CELLS / 32); g3 += blockDim.x >> 5) {
      const int cl = g3 * 32 + lane3;
      const int64_t key = key0 + cl;
      const int64_t first = a.start[key], end = a.start[key + 1];
      const int64_t P0 = __shfl_sync(0xffffffffu, first, 0);
      const int64_t P1 = __shfl_sync(0xffffffffu, end, 31);
      if (P0 >= P1) continue;
      const int l = cl & (TILE_CELLS - 1);
      const int ci = I0 + (l >> 6), cj = J0 + ((l >> 3) & 7),
                ck = K0 + (cl >> 9) * TILE + (l & 7);
      for (int64_t c0 = P0; c0 < P1; c0 += P2G_CH) {
        const int n = (int)(P1 - c0 < P2G_CH ? P1 - c0 : P2G_CH);
        __syncwarp();
        for (int i = lane3; i < n; i += 32) {
          const int64_t q = c0 + i;
          const float4 r0 = a.rec0[q], r1 = a.rec1[q];
          st[0 * P2G_CH + i] = div_dx(r0.x, dx, a.inv_dx_exact);
          st[1 * P2G_CH + i] = div_dx(r0.y, dx, a.inv_dx_exact);
          st[2 * P2G_CH + i] = div_dx(r0.z, dx, a.inv_dx_exact);
          if (APIC) {  // records 1..3: (v_c, C row c)
            const float4 r2 = a.rec2[q], r3 = a.rec3[q];
            const float f[15] = {r1.x, r2.x, r3.x, r0.x, r0.y, r0.z, r1.y, r1.z,
                                 r1.w, r2.y, r2.z, r2.w, r3.y, r3.z, r3.w};
#pragma unroll
            for (int m = 0; m < 15; ++m) st[(3 + m) * P2G_CH + i] = f[m];
          } else {
            st[3 * P2G_CH + i] = r1.x;
            st[4 * P2G_CH + i] = r1.y;
            st[5 * P2G_CH + i] = r1.z;
          }
        }
        __syncwarp();
        const int64_t lo64 = first > c0 ? first : c0, hi64 = end < c0 + n ? end : c0 + n;
        const int cnt = hi64 > lo64 ? (int)(hi64 - lo64) : 0;
        const int lo = (int)(lo64 - c0);
        const int maxcnt = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
        if (maxcnt == 0) continue;
        p2g_cell_comp_staged<APIC, KT, 0, T>(a, s_val, s_wt, st, lo, cnt, maxcnt, ci, cj, ck, I0,
                                             J0, K0);
        p2g_cell_comp_staged<APIC, KT, 1, T>(a, s_val + BK, s_wt + BK, st, lo, cnt, maxcnt, ci,
                                             cj, ck, I0, J0, K0);
        p2g_cell_comp_staged<APIC, KT, 2, T>(a, s_val + 2 * BK, s_wt + 2 * BK, st, lo, cnt,
                                             maxcnt, ci, cj, ck, I0, J0, K0);
      }
    }
    __syncthreads();
    p2g_flush_box<KT, T>(a, s_val, s_wt, I0, J0, K0);
    return;
  }
  if (MAP == 2) {
    const int lane2 = threadIdx.x & 31;
    for (int g2 = threadIdx.x >> 5; g2 < ntk * (TILE_CELLS / 32); g2 += blockDim.x >> 5) {
      const int cl = g2 * 32 + lane2;
      const int64_t key = key0 + cl;
      const int64_t first = a.start[key];
      const int cnt = (int)(a.start[key + 1] - first);
      const int maxcnt = (int)__reduce_max_sync(0xffffffffu, (unsigned)cnt);
      if (maxcnt == 0) continue;
      const int l = cl & (TILE_CELLS - 1);
      const int ci = I0 + (l >> 6), cj = J0 + ((l >> 3) & 7), ck = K0 + (cl >> 9) * TILE + (l & 7);
      p2g_cell_comp<APIC, KT, 0, T>(a, s_val, s_wt, first, cnt, maxcnt, ci, cj, ck, I0, J0, K0);
      p2g_cell_comp<APIC, KT, 1, T>(a, s_val + BK, s_wt + BK, first, cnt, maxcnt, ci, cj, ck, I0,
                                    J0, K0);
      p2g_cell_comp<APIC, KT, 2, T>(a, s_val + 2 * BK, s_wt + 2 * BK, first, cnt, maxcnt, ci, cj,
                                    ck, I0, J0, K0);
    }
    __syncthreads();
    p2g_flush_box<KT, T>(a, s_val, s_wt, I0, J0, K0);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int64_t np_tile = e - b, run = (np_tile + 31) >> 5;
  const int ngroups = MAP == 1 ? ntk * (TILE_CELLS / 32) : 0;
  int g = warp, kround = 0, cnt = 0;
  int64_t first = 0;
  if (MAP == 1 && g < ngroups) {
    const int64_t key = key0 + g * 32 + lane;
    first = a.start[key];
    cnt = (int)(a.start[key + 1] - first);
  }
  for (int64_t s = warp;; s += nwarps) {
    int64_t q;
    if (MAP == 0) {
      if (s >= run) break;
      const int64_t off = (int64_t)lane * run + s;
      if (off >= np_tile) continue;
      q = b + off;
    } else {
      // next (cell group, round) with work for this warp
      while (g < ngroups && kround >= __reduce_max_sync(0xffffffffu, (unsigned)cnt)) {
        g += nwarps;
        kround = 0;
        cnt = 0;
        if (g < ngroups) {
          const int64_t key = key0 + g * 32 + lane;
          first = a.start[key];
          cnt = (int)(a.start[key + 1] - first);
        }
      }
      if (g >= ngroups) break;
      const int kk = kround++;
      if (kk >= cnt) continue;
      q = first + kk;
    }
    float4 r0 = a.rec0[q], r1 = a.rec1[q];
    float4 r2 = make_float4(0, 0, 0, 0), r3 = r2;
    if (APIC) {
      r2 = a.rec2[q];
      r3 = a.rec3[q];
    }
    const float inv = a.inv_dx_exact;
    float gx = div_dx(r0.x, a.dx, inv), gy = div_dx(r0.y, a.dx, inv), gz = div_dx(r0.z, a.dx, inv);
    float hx = gx - 0.5f, hy = gy - 0.5f, hz = gz - 0.5f;
    // component c: velocity and C row.  APIC: record 1 + c holds (v_c, C row
    // c); FLIP/PIC: record 1 holds (vx, vy, vz)
    const float vc0 = r1.x, vc1 = APIC ? r2.x : r1.y, vc2 = APIC ? r3.x : r1.z;
    T *v0 = s_val, *w0 = s_wt, *v1 = s_val + BK, *w1 = s_wt + BK, *v2 = s_val + 2 * BK,
      *w2 = s_wt + 2 * BK;
    if (!scatter_comp_fast<APIC, KT, T>(v0, w0, 0, vc0, r1.y, r1.z, r1.w, r0.x, r0.y, r0.z, gx,
                                        hy, hz, I0, J0, K0, a))
      scatter_comp<APIC, KT, T>(v0, w0, 0, vc0, r1.y, r1.z, r1.w, r0.x, r0.y, r0.z, gx, hy, hz,
                                I0, J0, K0, a, a.u, a.uw);
    if (!scatter_comp_fast<APIC, KT, T>(v1, w1, 1, vc1, r2.y, r2.z, r2.w, r0.x, r0.y, r0.z, hx,
                                        gy, hz, I0, J0, K0, a))
      scatter_comp<APIC, KT, T>(v1, w1, 1, vc1, r2.y, r2.z, r2.w, r0.x, r0.y, r0.z, hx, gy, hz,
                                I0, J0, K0, a, a.v, a.vw);
    if (!scatter_comp_fast<APIC, KT, T>(v2, w2, 2, vc2, r3.y, r3.z, r3.w, r0.x, r0.y, r0.z, hx,
                                        hy, gz, I0, J0, K0, a))
      scatter_comp<APIC, KT, T>(v2, w2, 2, vc2, r3.y, r3.z, r3.w, r0.x, r0.y, r0.z, hx, hy, gz,
                                I0, J0, K0, a, a.w, a.ww);
  }
  __syncthreads();
  p2g_flush_box<KT, T>(a, s_val, s_wt, I0, J0, K0);
}

// Dynamic shared memory of a P2G block: the boxes, and for lane map 3 the
// staging areas of its 8 warps.
__host__ __device__ constexpr size_t p2g_smem_bytes(int KT, int map = 0, bool apic = true) {
  return 2 * 3 * (size_t)P2G_BOXK(KT) * sizeof(P2G_ACC) +
         (map == 3 ? (size_t)8 * p2g_stage_fields(apic) * P2G_CH * sizeof(float) : 0) +
         (map == 4 || map == 5
              ? (size_t)8 * (apic ? p2g_round_fields<true>() : p2g_round_fields<false>()) *
                    (map == 4 ? 8 : 4) * 32 * sizeof(float)
              : 0);
}

// One CTA per block of KT tiles along k: block b holds tiles (ti, tj, KT*kb
// .. KT*kb + KT - 1) with kb = b % ceil(ntz / KT), clipped to the grid.
#ifndef GF_P2G_MINB
#define GF_P2G_MINB 2  // resident CTAs per SM the register-summing map is compiled for
#endif
template <bool APIC, int KT, int MAP>
__global__ void __launch_bounds__(256, MAP >= 2 ? GF_P2G_MINB : 1) k_p2g_tile(P2GArgs a) {
  const int ntkb = (a.ntz + KT - 1) / KT;
  const int kb = blockIdx.x % ntkb, r = blockIdx.x / ntkb;
  const int t = r * a.ntz + KT * kb;  // r = ti * nty + tj
  const int ntk = a.ntz - KT * kb < KT ? a.ntz - KT * kb : KT;
  p2g_tile_body<APIC, KT, MAP>(a, t, (int64_t)t * TILE_CELLS, ntk);
}

// --------------------------------------------------------------- forces
struct GridArgs {
  float *u, *v, *w, *us, *vs, *ws;
  const float *uw, *vw, *ww;
  const uint8_t *label;
  const float *solid_u, *solid_v, *solid_w;
  float *div;
  const float *p;
  int nx, ny, nz;
};

// Face slot q = (i*(ny+1) + j)*(nz+1) + k carries the u, v and w faces (i,j,k)
// that exist.
// (i, j, k) of face slot q; 32-bit division when the slot count allows it
// (a 64-bit division is several times the instructions).
__device__ __forceinline__ void slot_ijk(int64_t q, int ny1, int nz1, bool small, int &i, int &j,
                                         int &k) {
  if (small) {
    const uint32_t u = (uint32_t)q, r = u / (uint32_t)nz1;
    k = (int)(u - r * (uint32_t)nz1);
    j = (int)(r % (uint32_t)ny1);
    i = (int)(r / (uint32_t)ny1);
  } else {
    k = (int)(q % nz1);
    const int64_t r = q / nz1;
    j = (int)(r % ny1);
    i = (int)(r / ny1);
  }
}

__device__ __forceinline__ void forces_slot(const GridArgs &a, int64_t q, float gd,
                                            bool small = false) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  {
    int i, j, k;
    slot_ijk(q, ny + 1, nz + 1, small, i, j, k);
    if (j < ny && k < nz) {  // u face (i,j,k), i <= nx
      int64_t g = ((int64_t)i * ny + j) * nz + k;
      float wt = a.uw[g];
      float val = wt > 1.0e-8f ? a.u[g] / wt : 0.0f;
      a.us[g] = val;
      bool left = i == 0 || a.label[((int64_t)(i - 1) * ny + j) * nz + k] == 2;
      bool right = i == nx || a.label[((int64_t)i * ny + j) * nz + k] == 2;
      if (left || right) val = a.solid_u ? a.solid_u[g] : 0.0f;
      a.u[g] = val;
    }
    if (i < nx && k < nz) {  // v face (i,j,k), j <= ny
      int64_t g = ((int64_t)i * (ny + 1) + j) * nz + k;
      float wt = a.vw[g];
      float val = wt > 1.0e-8f ? a.v[g] / wt : 0.0f;
      a.vs[g] = val;
      val = val + gd;  // gravity on every v face (:149-156)
      bool bot = j == 0 || a.label[((int64_t)i * ny + (j - 1)) * nz + k] == 2;
      bool top = j == ny || a.label[((int64_t)i * ny + j) * nz + k] == 2;
      if (bot || top) val = a.solid_v ? a.solid_v[g] : 0.0f;
      a.v[g] = val;
    }
    if (i < nx && j < ny) {  // w face (i,j,k), k <= nz
      int64_t g = ((int64_t)i * ny + j) * (nz + 1) + k;
      float wt = a.ww[g];
      float val = wt > 1.0e-8f ? a.w[g] / wt : 0.0f;
      a.ws[g] = val;
      bool back = k == 0 || a.label[((int64_t)i * ny + j) * nz + (k - 1)] == 2;
      bool front = k == nz || a.label[((int64_t)i * ny + j) * nz + k] == 2;
      if (back || front) val = a.solid_w ? a.solid_w[g] : 0.0f;
      a.w[g] = val;
    }
  }
}

__global__ void k_forces(GridArgs a, float gd) {
  int64_t n = (int64_t)(a.nx + 1) * (a.ny + 1) * (a.nz + 1);
  const bool small = n < ((int64_t)1 << 32);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    forces_slot(a, q, gd, small);
}

__device__ __forceinline__ void divergence_cell(const GridArgs &a, int64_t c, float scale,
                                                bool small = false) {
  const int ny = a.ny, nz = a.nz;
  {
    if (a.label[c] != 1) {
      a.div[c] = 0.0f;
      return;
    }
    int i, j, k;
    slot_ijk(c, ny, nz, small, i, j, k);
    float d = a.u[((int64_t)(i + 1) * ny + j) * nz + k] - a.u[c];
    d = d + a.v[((int64_t)i * (ny + 1) + j + 1) * nz + k];
    d = d - a.v[((int64_t)i * (ny + 1) + j) * nz + k];
    d = d + a.w[((int64_t)i * ny + j) * (nz + 1) + k + 1];
    d = d - a.w[((int64_t)i * ny + j) * (nz + 1) + k];
    a.div[c] = d * scale;
  }
}

__global__ void k_divergence(GridArgs a, float scale) {
  int64_t n = (int64_t)a.nx * a.ny * a.nz;
  const bool small = n < ((int64_t)1 << 32);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    divergence_cell(a, c, scale, small);
}

__device__ __forceinline__ void project_slot(const GridArgs &a, int64_t q, float scale,
                                             bool small = false) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  {
    int i, j, k;
    slot_ijk(q, ny + 1, nz + 1, small, i, j, k);
    const int64_t c = ((int64_t)i * ny + j) * nz + k;  // valid when i<nx,j<ny,k<nz
    if (j < ny && k < nz) {  // u face
      int64_t g = ((int64_t)i * ny + j) * nz + k;
      float val = a.u[g];
      if (i >= 1 && i <= nx - 1) {
        int ml = a.label[c - (int64_t)ny * nz], mr = a.label[c];
        if ((ml == 1 || mr == 1) && ml != 2 && mr != 2) {
          float pl = ml == 1 ? a.p[c - (int64_t)ny * nz] : 0.0f;
          float pr = mr == 1 ? a.p[c] : 0.0f;
          float gr = pr - pl;
          gr = scale * gr;
          val = val - gr;
        }
      }
      bool left = i == 0 || a.label[c - (int64_t)ny * nz] == 2;
      bool right = i == nx || a.label[c] == 2;
      if (left || right) val = a.solid_u ? a.solid_u[g] : 0.0f;
      a.u[g] = val;
    }
    if (i < nx && k < nz) {  // v face
      int64_t g = ((int64_t)i * (ny + 1) + j) * nz + k;
      float val = a.v[g];
      if (j >= 1 && j <= ny - 1) {
        int mb = a.label[c - nz], mt = a.label[c];
        if ((mb == 1 || mt == 1) && mb != 2 && mt != 2) {
          float pb = mb == 1 ? a.p[c - nz] : 0.0f;
          float pt = mt == 1 ? a.p[c] : 0.0f;
          float gr = pt - pb;
          gr = scale * gr;
          val = val - gr;
        }
      }
      bool bot = j == 0 || a.label[c - nz] == 2;
      bool top = j == ny || a.label[c] == 2;
      if (bot || top) val = a.solid_v ? a.solid_v[g] : 0.0f;
      a.v[g] = val;
    }
    if (i < nx && j < ny) {  // w face
      int64_t g = ((int64_t)i * ny + j) * (nz + 1) + k;
      float val = a.w[g];
      if (k >= 1 && k <= nz - 1) {
        int mba = a.label[c - 1], mfr = a.label[c];
        if ((mba == 1 || mfr == 1) && mba != 2 && mfr != 2) {
          float pba = mba == 1 ? a.p[c - 1] : 0.0f;
          float pfr = mfr == 1 ? a.p[c] : 0.0f;
          float gr = pfr - pba;
          gr = scale * gr;
          val = val - gr;
        }
      }
      bool back = k == 0 || a.label[c - 1] == 2;
      bool front = k == nz || a.label[c] == 2;
      if (back || front) val = a.solid_w ? a.solid_w[g] : 0.0f;
      a.w[g] = val;
    }
  }
}

__global__ void k_project(GridArgs a, float scale) {
  int64_t n = (int64_t)(a.nx + 1) * (a.ny + 1) * (a.nz + 1);
  const bool small = n < ((int64_t)1 << 32);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
       q += (int64_t)gridDim.x * blockDim.x)
    project_slot(a, q, scale, small);
}

// ------------------------------------------------------------------- G2P
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
  return x < lo ? lo : (x > hi ? hi : x);
}

// Face-array accessors of the G2P gathers: the array in global memory, or a
// staged box of it in shared memory (origin oi, oj, ok; nj x nk per i-plane).
struct GlobalAt {
  const float *__restrict__ f;
  int64_t si, sj;
  int64_t n;  // elements of the array (checked in the bounds-checked build)
  __device__ __forceinline__ float operator()(int i, int j, int k) const {
    const int64_t q = (int64_t)i * si + (int64_t)j * sj + k;
    return GF_IN(q, n) ? __ldg(f + q) : 0.0f;
  }
};
struct BoxAt {
  const float *s;
  int oi, oj, ok, nj, nk, vol;
  __device__ __forceinline__ float operator()(int i, int j, int k) const {
    const int q = ((i - oi) * nj + (j - oj)) * nk + (k - ok);
    return GF_IN(q, vol) ? s[q] : 0.0f;
  }
};

// sample3, gridmath.py:29-63 (clamped coordinates, clamped indices).
__device__ __forceinline__ void sample3_index(float &fx, float &fy, float &fz, int nxm, int nym,
                                              int nzm, int &i0, int &j0, int &k0, int &i1,
                                              int &j1, int &k1) {
  fx = clampf(fx, 0.0f, (float)nxm);
  fy = clampf(fy, 0.0f, (float)nym);
  fz = clampf(fz, 0.0f, (float)nzm);
  i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)), k0 = __float2int_rz(floorf(fz));
  if (i0 >= nxm) i0 = nxm - 1;
  if (j0 >= nym) j0 = nym - 1;
  if (k0 >= nzm) k0 = nzm - 1;
  if (i0 < 0) i0 = 0;
  if (j0 < 0) j0 = 0;
  if (k0 < 0) k0 = 0;
  i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  if (i1 >= nxm) i1 = nxm - 1;
  if (j1 >= nym) j1 = nym - 1;
  if (k1 >= nzm) k1 = nzm - 1;
}

template <class F>
__device__ __forceinline__ float sample3_at(const F &at, float fx, float fy, float fz, int i0,
                                            int j0, int k0, int i1, int j1, int k1) {
  float sx = clampf(fx - (float)i0, 0.0f, 1.0f);
  float sy = clampf(fy - (float)j0, 0.0f, 1.0f);
  float sz = clampf(fz - (float)k0, 0.0f, 1.0f);
  float c000 = at(i0, j0, k0), c100 = at(i1, j0, k0);
  float c010 = at(i0, j1, k0), c110 = at(i1, j1, k0);
  float c001 = at(i0, j0, k1), c101 = at(i1, j0, k1);
  float c011 = at(i0, j1, k1), c111 = at(i1, j1, k1);
  float ox = 1.0f - sx, oy = 1.0f - sy, oz = 1.0f - sz;
  float c00 = c000 * ox + c100 * sx;
  float c10 = c010 * ox + c110 * sx;
  float c01 = c001 * ox + c101 * sx;
  float c11 = c011 * ox + c111 * sx;
  float c0 = c00 * oy + c10 * sy;
  float c1 = c01 * oy + c11 * sy;
  return c0 * oz + c1 * sz;
}

// sample3_at for corners that needed no clamp (i1 = i0 + 1, j1 = j0 + 1,
// k1 = k0 + 1): corner (di, dj, dk) is element di*si + dj*sj + dk of `p`; the
// same products and sums in the same order.
__device__ __forceinline__ float sample3_lin(const float *p, int si, int sj, float fx, float fy,
                                             float fz, int i0, int j0, int k0) {
  float sx = clampf(fx - (float)i0, 0.0f, 1.0f);
  float sy = clampf(fy - (float)j0, 0.0f, 1.0f);
  float sz = clampf(fz - (float)k0, 0.0f, 1.0f);
  float c000 = p[0], c100 = p[si];
  float c010 = p[sj], c110 = p[si + sj];
  float c001 = p[1], c101 = p[si + 1];
  float c011 = p[sj + 1], c111 = p[si + sj + 1];
  float ox = 1.0f - sx, oy = 1.0f - sy, oz = 1.0f - sz;
  float c00 = c000 * ox + c100 * sx;
  float c10 = c010 * ox + c110 * sx;
  float c01 = c001 * ox + c101 * sx;
  float c11 = c011 * ox + c111 * sx;
  float c0 = c00 * oy + c10 * sy;
  float c1 = c01 * oy + c11 * sy;
  return c0 * oz + c1 * sz;
}

__device__ __forceinline__ float sample3(const float *__restrict__ f, float fx, float fy,
                                         float fz, int nxm, int nym, int nzm) {
  int i0, j0, k0, i1, j1, k1;
  sample3_index(fx, fy, fz, nxm, nym, nzm, i0, j0, k0, i1, j1, k1);
  if (i1 == i0 + 1 && j1 == j0 + 1 && k1 == k0 + 1)
    return sample3_lin(f + ((int64_t)i0 * nym + j0) * nzm + k0, nym * nzm, nzm, fx, fy, fz, i0,
                       j0, k0);
  return sample3_at(GlobalAt{f, (int64_t)nym * nzm, nzm, (int64_t)nxm * nym * nzm}, fx, fy, fz,
                    i0, j0, k0, i1, j1, k1);
}

// One face component of k3_g2p_apic_advect (:1626-1724): clamped-index
// gather of velocity and of the C row.
template <class F>
__device__ __forceinline__ void apic_gather_at(const F &at, float px, float py, float pz,
                                               float dx, float fx, float fy, float fz, int snx,
                                               int sny, int snz, int ax, float inv, float &vel,
                                               float &c0, float &c1, float &c2) {
  int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
      k0 = __float2int_rz(floorf(fz));
  float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  float acc = 0.0f;
  c0 = 0.0f;
  c1 = 0.0f;
  c2 = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        int ii = i0 + di, jj = j0 + dj, kk = k0 + dk;
        if (ii < 0) ii = 0;
        if (jj < 0) jj = 0;
        if (kk < 0) kk = 0;
        if (ii > snx - 1) ii = snx - 1;
        if (jj > sny - 1) jj = sny - 1;
        if (kk > snz - 1) kk = snz - 1;
        float wxi = di == 0 ? 1.0f - sx : sx;
        float wyi = dj == 0 ? 1.0f - sy : sy;
        float wzi = dk == 0 ? 1.0f - sz : sz;
        float wt = wxi * wyi;
        wt = wt * wzi;
        float val = at(ii, jj, kk);
        float t = wt * val;
        acc = acc + t;
        float ox = ax == 0 ? (float)ii * dx - px : ((float)ii + 0.5f) * dx - px;
        float oy = ax == 1 ? (float)jj * dx - py : ((float)jj + 0.5f) * dx - py;
        float oz = ax == 2 ? (float)kk * dx - pz : ((float)kk + 0.5f) * dx - pz;
        float fu = t * inv;
        c0 = c0 + fu * ox;
        c1 = c1 + fu * oy;
        c2 = c2 + fu * oz;
      }
  vel = acc;
}

// apic_gather_at when no index needs clamping (every corner inside the
// component's grid): the corner (di, dj, dk) is element di*si + dj*sj + dk of
// `p` (the stencil's first corner), and the per-axis face offsets and the
// products wx * wy are formed once.  Every product and sum is the one
// apic_gather_at forms, in the same order, so the results are identical;
// only the index arithmetic (the clamps, one address per corner) is gone.
__device__ __forceinline__ void apic_gather_lin(const float *p, int si, int sj, int i0, int j0,
                                                int k0, float px, float py, float pz, float dx,
                                                float fx, float fy, float fz, int ax, float inv,
                                                float &vel, float &c0, float &c1, float &c2) {
  const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
  float ox[2], oy[2], oz[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    ox[d] = ax == 0 ? (float)(i0 + d) * dx - px : ((float)(i0 + d) + 0.5f) * dx - px;
    oy[d] = ax == 1 ? (float)(j0 + d) * dx - py : ((float)(j0 + d) + 0.5f) * dx - py;
    oz[d] = ax == 2 ? (float)(k0 + d) * dx - pz : ((float)(k0 + d) + 0.5f) * dx - pz;
  }
  float acc = 0.0f;
  c0 = 0.0f;
  c1 = 0.0f;
  c2 = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const float wxy = wx[di] * wy[dj];
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const float wt = wxy * wz[dk];
        const float t = wt * p[di * si + dj * sj + dk];
        acc = acc + t;
        const float fu = t * inv;
        c0 = c0 + fu * ox[di];
        c1 = c1 + fu * oy[dj];
        c2 = c2 + fu * oz[dk];
      }
    }
  vel = acc;
}

// Stencil of one component for the paired gathers: its first corner in the
// staged box, the box strides, the first face index per axis and the sample
// coordinates.
struct GStencil {
  const float *p;
  int si, sj, i0, j0, k0;
  float fx, fy, fz;
  float i0f, j0f, k0f;  // floor(fx), ...: the first face indices as floats (exact)
};

// apic_gather_lin for two components at once (a on the x half of each
// float32 pair, b on the y half): every product and sum is the one
// apic_gather_lin forms for that component, in the same order, done by the
// paired f32x2 instructions (each half rounds as the scalar operation), so
// both results are identical to two apic_gather_lin calls.  A sum that takes
// a product is formed as fma(x, one, y) with one == 1 known only at run time
// (sum2): the compiler contracts a paired product into a paired add even with
// contraction disabled, which would round the two operations once.
template <int AXA, int AXB>
__device__ __forceinline__ void apic_gather_lin_pair(const GStencil &a, const GStencil &b,
                                                     float px, float py, float pz, float dx,
                                                     float inv, float one, float2 &vel,
                                                     float2 &c0, float2 &c1, float2 &c2) {
  const float2 ONE = dup2(one), NEG = dup2(-one);
  // first face indices as floats: float(floor(f)) is floor(f), and adding 1
  // to it is exact, so no integer-to-float conversion is needed
  const float2 I0[2] = {make_float2(a.i0f, b.i0f), add2(make_float2(a.i0f, b.i0f), dup2(1.0f))};
  const float2 J0[2] = {make_float2(a.j0f, b.j0f), add2(make_float2(a.j0f, b.j0f), dup2(1.0f))};
  const float2 K0[2] = {make_float2(a.k0f, b.k0f), add2(make_float2(a.k0f, b.k0f), dup2(1.0f))};
  // s = f - floor(f): the difference as -floor * 1 + f
  const float2 s_x = fma2(I0[0], NEG, make_float2(a.fx, b.fx));
  const float2 s_y = fma2(J0[0], NEG, make_float2(a.fy, b.fy));
  const float2 s_z = fma2(K0[0], NEG, make_float2(a.fz, b.fz));
  const float2 wx[2] = {sub2(dup2(1.0f), s_x), s_x}, wy[2] = {sub2(dup2(1.0f), s_y), s_y},
               wz[2] = {sub2(dup2(1.0f), s_z), s_z};
  // face offsets: (index [+ 0.5]) dx - p; adding 0 to the integer-valued float
  // is exact, so the component without the half shift keeps its value
  const float2 hx = make_float2(AXA == 0 ? 0.0f : 0.5f, AXB == 0 ? 0.0f : 0.5f);
  const float2 hy = make_float2(AXA == 1 ? 0.0f : 0.5f, AXB == 1 ? 0.0f : 0.5f);
  const float2 hz = make_float2(AXA == 2 ? 0.0f : 0.5f, AXB == 2 ? 0.0f : 0.5f);
  const float2 DX = dup2(dx);
  float2 ox[2], oy[2], oz[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    ox[d] = sum2(mul2(add2(I0[d], hx), DX), ONE, dup2(-px));
    oy[d] = sum2(mul2(add2(J0[d], hy), DX), ONE, dup2(-py));
    oz[d] = sum2(mul2(add2(K0[d], hz), DX), ONE, dup2(-pz));
  }
  const float2 INV = dup2(inv);
  float2 acc = dup2(0.0f);
  c0 = c1 = c2 = dup2(0.0f);
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const float2 wxy = mul2(wx[di], wy[dj]);
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const float2 wt = mul2(wxy, wz[dk]);
        const float2 val = make_float2(a.p[di * a.si + dj * a.sj + dk],
                                       b.p[di * b.si + dj * b.sj + dk]);
        const float2 t = mul2(wt, val);
        acc = sum2(t, ONE, acc);
        const float2 fu = mul2(t, INV);
        c0 = sum2(mul2(fu, ox[di]), ONE, c0);
        c1 = sum2(mul2(fu, oy[dj]), ONE, c1);
        c2 = sum2(mul2(fu, oz[dk]), ONE, c2);
      }
    }
  vel = acc;
}

// apic_gather_lin for one component with its two corners along k paired:
// the products of both corners are paired f32x2 instructions, and each
// accumulator adds the dk = 0 term before the dk = 1 term, as
// apic_gather_lin does, so the results are identical (the paired sum that
// takes a product is a sum2, as in apic_gather_lin_pair).
template <int AX>
__device__ __forceinline__ void apic_gather_lin_k2(const GStencil &g, float px, float py,
                                                   float pz, float dx, float inv, float one,
                                                   float &vel, float &c0, float &c1, float &c2) {
  const float sx = g.fx - g.i0f, sy = g.fy - g.j0f, sz = g.fz - g.k0f;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy};
  const float2 wz = make_float2(1.0f - sz, sz);
  float ox[2], oy[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {  // float(i0 + d) as floor + d (exact)
    const float fi = g.i0f + (float)d, fj = g.j0f + (float)d;
    ox[d] = AX == 0 ? fi * dx - px : (fi + 0.5f) * dx - px;
    oy[d] = AX == 1 ? fj * dx - py : (fj + 0.5f) * dx - py;
  }
  const float2 oz = sum2(mul2(add2(make_float2(g.k0f, g.k0f + 1.0f),
                                   dup2(AX == 2 ? 0.0f : 0.5f)),
                              dup2(dx)),
                         dup2(one), dup2(-pz));
  const float2 INV = dup2(inv);
  float acc = 0.0f;
  c0 = 0.0f;
  c1 = 0.0f;
  c2 = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      const float wxy = wx[di] * wy[dj];
      const float *q = g.p + di * g.si + dj * g.sj;
      const float2 wt = mul2(dup2(wxy), wz);
      const float2 t = mul2(wt, make_float2(q[0], q[1]));
      const float2 fu = mul2(t, INV);
      const float2 m0 = mul2(fu, dup2(ox[di])), m1 = mul2(fu, dup2(oy[dj])), m2 = mul2(fu, oz);
      acc = acc + t.x;
      c0 = c0 + m0.x;
      c1 = c1 + m1.x;
      c2 = c2 + m2.x;
      acc = acc + t.y;
      c0 = c0 + m0.y;
      c1 = c1 + m1.y;
      c2 = c2 + m2.y;
    }
  vel = acc;
}

// sample3_lin of two arrays that share the stencil (the new and the saved
// velocity of one component): the weights are formed once and every
// interpolation step is a paired f32x2 instruction (x half: p, y half: q),
// each half rounding as sample3_lin's scalar step, so both results are
// identical to two sample3_lin calls (sums of products are sum2s, as in
// apic_gather_lin_pair).
__device__ __forceinline__ float2 sample3_lin_pair(const float *p, const float *q, int si,
                                                   int sj, float fx, float fy, float fz, int i0,
                                                   int j0, int k0, float one) {
  const float sx = clampf(fx - (float)i0, 0.0f, 1.0f);
  const float sy = clampf(fy - (float)j0, 0.0f, 1.0f);
  const float sz = clampf(fz - (float)k0, 0.0f, 1.0f);
  const float2 SX = dup2(sx), SY = dup2(sy), SZ = dup2(sz), ONE = dup2(one);
  const float2 OX = dup2(1.0f - sx), OY = dup2(1.0f - sy), OZ = dup2(1.0f - sz);
  const float2 c000 = make_float2(p[0], q[0]), c100 = make_float2(p[si], q[si]);
  const float2 c010 = make_float2(p[sj], q[sj]), c110 = make_float2(p[si + sj], q[si + sj]);
  const float2 c001 = make_float2(p[1], q[1]), c101 = make_float2(p[si + 1], q[si + 1]);
  const float2 c011 = make_float2(p[sj + 1], q[sj + 1]);
  const float2 c111 = make_float2(p[si + sj + 1], q[si + sj + 1]);
  const float2 c00 = sum2(mul2(c000, OX), ONE, mul2(c100, SX));
  const float2 c10 = sum2(mul2(c010, OX), ONE, mul2(c110, SX));
  const float2 c01 = sum2(mul2(c001, OX), ONE, mul2(c101, SX));
  const float2 c11 = sum2(mul2(c011, OX), ONE, mul2(c111, SX));
  const float2 c0 = sum2(mul2(c00, OY), ONE, mul2(c10, SY));
  const float2 c1 = sum2(mul2(c01, OY), ONE, mul2(c11, SY));
  return sum2(mul2(c0, OZ), ONE, mul2(c1, SZ));
}

// True when apic_gather_at's stencil at (fx, fy, fz) needs no clamp.
__device__ __forceinline__ bool stencil_inside(float fx, float fy, float fz, int snx, int sny,
                                               int snz, int &i0, int &j0, int &k0) {
  i0 = __float2int_rz(floorf(fx));
  j0 = __float2int_rz(floorf(fy));
  k0 = __float2int_rz(floorf(fz));
  return i0 >= 0 && i0 < snx - 1 && j0 >= 0 && j0 < sny - 1 && k0 >= 0 && k0 < snz - 1;
}

__device__ __forceinline__ void apic_gather(const float *__restrict__ f, float px, float py,
                                            float pz, float dx, float fx, float fy, float fz,
                                            int snx, int sny, int snz, int ax, float inv,
                                            float &vel, float &c0, float &c1, float &c2) {
  int i0, j0, k0;
  if (stencil_inside(fx, fy, fz, snx, sny, snz, i0, j0, k0))
    apic_gather_lin(f + ((int64_t)i0 * sny + j0) * snz + k0, sny * snz, snz, i0, j0, k0, px, py,
                    pz, dx, fx, fy, fz, ax, inv, vel, c0, c1, c2);
  else
    apic_gather_at(GlobalAt{f, (int64_t)sny * snz, snz, (int64_t)snx * sny * snz}, px, py, pz,
                   dx, fx, fy, fz, snx, sny, snz, ax, inv, vel, c0, c1, c2);
}

struct G2PArgs {
  const float4 *rec0, *rec1;
  const float *u, *v, *w, *us, *vs, *ws;
  float *pos, *vel, *C;
  int32_t *pid;
  int64_t n;
  float dx, dt, flip_blend, dom0, dom1, dom2;
  int nx, ny, nz;
  float inv_dx_exact;  // exact_inverse(dx)
  float one = 1.0f;    // 1, as a launch argument (sum2's multiplier)
};

template <bool APIC>
__device__ __forceinline__ void g2p_particle(const G2PArgs &a, int64_t q) {
  const float4 r0 = a.rec0[q];
  const float px = r0.x, py = r0.y, pz = r0.z;
  const float dx = a.dx, idx = a.inv_dx_exact;
  float gx = div_dx(px, dx, idx), gy = div_dx(py, dx, idx), gz = div_dx(pz, dx, idx);
  float hx = gx - 0.5f, hy = gy - 0.5f, hz = gz - 0.5f;
  float nu, nv, nw;
  if (APIC) {
    float dd = dx * dx;
    float inv = __fdiv_rn(3.0f, dd);
    float c[9];
    apic_gather(a.u, px, py, pz, dx, gx, hy, hz, a.nx + 1, a.ny, a.nz, 0, inv, nu, c[0], c[1], c[2]);
    apic_gather(a.v, px, py, pz, dx, hx, gy, hz, a.nx, a.ny + 1, a.nz, 1, inv, nv, c[3], c[4], c[5]);
    apic_gather(a.w, px, py, pz, dx, hx, hy, gz, a.nx, a.ny, a.nz + 1, 2, inv, nw, c[6], c[7], c[8]);
#pragma unroll
    for (int m = 0; m < 9; ++m) a.C[9 * q + m] = c[m];
  } else {
    const float4 r1 = a.rec1[q];
    float pic_u = sample3(a.u, gx, hy, hz, a.nx + 1, a.ny, a.nz);
    float old_u = sample3(a.us, gx, hy, hz, a.nx + 1, a.ny, a.nz);
    float pic_v = sample3(a.v, hx, gy, hz, a.nx, a.ny + 1, a.nz);
    float old_v = sample3(a.vs, hx, gy, hz, a.nx, a.ny + 1, a.nz);
    float pic_w = sample3(a.w, hx, hy, gz, a.nx, a.ny, a.nz + 1);
    float old_w = sample3(a.ws, hx, hy, gz, a.nx, a.ny, a.nz + 1);
    float fu = r1.x + (pic_u - old_u), fv = r1.y + (pic_v - old_v), fw = r1.z + (pic_w - old_w);
    float ob = 1.0f - a.flip_blend;
    nu = a.flip_blend * fu + ob * pic_u;
    nv = a.flip_blend * fv + ob * pic_v;
    nw = a.flip_blend * fw + ob * pic_w;
  }
  a.vel[3 * q] = nu;
  a.vel[3 * q + 1] = nv;
  a.vel[3 * q + 2] = nw;
  const float eps = dx * 1.001f;
  a.pos[3 * q] = clampf(px + nu * a.dt, eps, a.dom0 - eps);
  a.pos[3 * q + 1] = clampf(py + nv * a.dt, eps, a.dom1 - eps);
  a.pos[3 * q + 2] = clampf(pz + nw * a.dt, eps, a.dom2 - eps);
  a.pid[q] = __float_as_int(r0.w);
}

template <bool APIC>
__global__ void __launch_bounds__(512) k_g2p(G2PArgs a) {
  int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= a.n) return;
  g2p_particle<APIC>(a, q);
}

// ------------------------------------------------------- G2P, tile-staged
// k_g2p_tile: CTAs per 8x8x8 tile (or 8x8x16 block) of the cell-sorted
// particles, up to G2P_SPLIT_N particles each.  The faces
// the tile's particles can gather -- per component a box of 9 faces on its
// normal axis and 10 on the transverse axes around the tile -- are staged in
// shared memory first: by TMA (cp.async.bulk.tensor, completion on an
// mbarrier) for every face array whose layout admits a tensor map, by plain
// loads for the others.  The gathers then read shared memory, and the
// outputs (positions, velocities, C, ids; AoS) go through a per-warp shared
// staging buffer, so that each warp store instruction writes 32 consecutive
// floats of one array (no block barrier between rounds).
// The arithmetic is that of k_g2p, operation for operation.
//
// Box of component c (0 u, 1 v, 2 w) at tile origin (I0, J0, K0), in face
// indices: i from oi = I0 - (c != 0) over gbox_ni(c) planes, j from
// oj = J0 - (c != 1) over gbox_nj(c) rows, k from ok over gbox_nk(c): u and v
// need k in [K0-1, K0+8] and load [K0-4, K0+12), w needs [K0, K0+8] and loads
// [K0, K0+12) -- the start and width of the innermost axis are multiples of
// 16 bytes, as a tiled TMA copy requires.  Boxes start on 128-byte
// boundaries; a set of three boxes (u, v, w) takes GBOX_SET floats.
// With KT tiles per block along k (the autotuner's tile shape) the k ranges
// grow by 8 (KT - 1): u and v load [K0-4, K0+8KT+4), w [K0, K0+8KT+4).
__host__ __device__ constexpr int gbox_ni(int c) { return c == 0 ? 9 : 10; }
__host__ __device__ constexpr int gbox_nj(int c) { return c == 1 ? 9 : 10; }
__host__ __device__ constexpr int gbox_nk(int c, int KT = 1) {
  return c == 2 ? 8 * KT + 4 : 8 * KT + 8;
}
__host__ __device__ constexpr int gbox_vol(int c, int KT = 1) {
  return gbox_ni(c) * gbox_nj(c) * gbox_nk(c, KT);
}
__host__ __device__ constexpr int align32(int v) { return (v + 31) & ~31; }  // 128 bytes
__host__ __device__ constexpr int gbox_off(int c, int KT = 1) {
  return c == 0 ? 0
                : (c == 1 ? align32(gbox_vol(0, KT))
                          : align32(gbox_vol(0, KT)) + align32(gbox_vol(1, KT)));
}
__host__ __device__ constexpr int gbox_set(int KT) {
  return align32(gbox_off(2, KT) + gbox_vol(2, KT));
}
constexpr int GBOX_SET = 4096;
static_assert(gbox_vol(0) == 1440 && gbox_vol(1) == 1440 && gbox_vol(2) == 1200, "boxes");
static_assert(gbox_off(2) == 2880 && gbox_set(1) == GBOX_SET, "box set");
static_assert(gbox_set(2) == 6368, "box set of 8 x 8 x 16 blocks");
constexpr int G2P_TILE_THREADS = 256;
constexpr int G2P_SPLIT_N = 2048;  // particles per CTA (8 rounds of 256)
constexpr int G2P_SPLITS = 2;      // CTAs per 8^3 tile: 4096 particles at 8 per cell
constexpr long long G2P_WAIT_LIMIT = 1LL << 22;  // try_wait polls before giving up

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Tiled 3-D TMA load of one box into this CTA's shared memory (no multicast).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

struct G2PTileArgs {
  G2PArgs g;
  const int32_t *start;
  int nty, ntz;
  int32_t *wait_err;  // incremented when the box loads do not complete in time
};

__host__ __device__ constexpr size_t g2p_smem_bytes(int mode, int KT) {
  return (size_t)(mode == GF_APIC ? 1 : 2) * gbox_set(KT) * sizeof(float);
}

// True when the clamped gather indices [lo, hi] of every axis lie inside the
// component's box (always, for a particle inside its binned cell; a particle
// outside the grid or with a non-finite position takes the global path).
__device__ __forceinline__ bool in_box(const BoxAt &b, int ni, int i0, int i1, int j0, int j1,
                                       int k0, int k1) {
  return i0 >= b.oi && i1 < b.oi + ni && j0 >= b.oj && j1 < b.oj + b.nj && k0 >= b.ok &&
         k1 < b.ok + b.nk;
}

template <int MODE, int KT>
__global__ void __launch_bounds__(G2P_TILE_THREADS, 4)
    k_g2p_tile(const G2PTileArgs ta, const __grid_constant__ FaceMaps fm) {
  constexpr bool APIC = MODE == GF_APIC;
  constexpr int NARR = APIC ? 3 : 6;  // u, v, w (+ us, vs, ws for the FLIP delta)
  // output staging, per warp: pos 96, vel 96, [C 288,] pid 32 floats
  constexpr int PW = APIC ? 512 : 224, OUTF = 8 * PW;
  static_assert(G2P_TILE_THREADS == 256, "eight warps of staging");
  constexpr int SET = gbox_set(KT);
  extern __shared__ __align__(128) unsigned char g2p_smem[];
  float *s_box = reinterpret_cast<float *>(g2p_smem);  // (NARR / 3) sets of boxes
  __shared__ alignas(16) float s_out[OUTF];
  __shared__ alignas(8) uint64_t s_bar;
  __shared__ int s_ok;
  const G2PArgs &a = ta.g;
  const int tid = threadIdx.x;
  // CTA -> (block of KT tiles along k, clipped at the grid's last tile; part
  // of the block's particles): G2P_SPLIT_N particles per CTA, the last part
  // taking whatever a crowded block holds beyond, so the work is spread over
  // many more CTAs than blocks
  constexpr int S = G2P_SPLITS * KT;
  const int sidx = blockIdx.x % S, blk = blockIdx.x / S;
  const int ntkb = (ta.ntz + KT - 1) / KT;
  const int kb = blk % ntkb, rij = blk / ntkb;
  const int t = rij * ta.ntz + KT * kb;
  const int ntk = ta.ntz - KT * kb < KT ? ta.ntz - KT * kb : KT;
  const int64_t b0 = ta.start[(int64_t)t * TILE_CELLS],
                e0 = ta.start[(int64_t)(t + ntk) * TILE_CELLS];
  const int64_t b = b0 + (int64_t)sidx * G2P_SPLIT_N;
  const int64_t e = sidx == S - 1 ? e0 : (b + G2P_SPLIT_N < e0 ? b + G2P_SPLIT_N : e0);
  if (b >= e) return;
  const int ti = rij / ta.nty, tj = rij % ta.nty;
  const int I0 = ti * TILE, J0 = tj * TILE, K0 = KT * kb * TILE;
  const int nx = a.nx, ny = a.ny, nz = a.nz;

  // ---- stage the boxes
  uint32_t tx = 0;
#pragma unroll
  for (int q = 0; q < NARR; ++q)
    if ((fm.mask >> q) & 1) tx += (uint32_t)gbox_vol(q % 3, KT) * 4u;
  if (tid == 0) {
    s_ok = 1;
    if (tx) {
      mbar_init(&s_bar, 1);
      mbar_init_fence();
    }
  }
  __syncthreads();
  if (tid == 0 && tx) {
    mbar_expect_tx(&s_bar, tx);
#pragma unroll
    for (int q = 0; q < NARR; ++q) {
      if (!((fm.mask >> q) & 1)) continue;
      const int c = q % 3;
      tma_load_3d(s_box + (q / 3) * SET + gbox_off(c, KT), &fm.m[q], c == 2 ? K0 : K0 - 4,
                  J0 - (c != 1), I0 - (c != 0), &s_bar);
    }
  }
  {
    const float *src[6] = {a.u, a.v, a.w, a.us, a.vs, a.ws};
#pragma unroll
    for (int q = 0; q < NARR; ++q) {
      if ((fm.mask >> q) & 1) continue;
      const int c = q % 3;
      const int snx = nx + (c == 0), sny = ny + (c == 1), snz = nz + (c == 2);
      const int ni = gbox_ni(c), nj = gbox_nj(c), nk = gbox_nk(c, KT);
      const int oi = I0 - (c != 0), oj = J0 - (c != 1), ok = c == 2 ? K0 : K0 - 4;
      float *dst = s_box + (q / 3) * SET + gbox_off(c, KT);
      // one thread per row of nk faces along k: the row's address once, then
      // nk consecutive loads (zero outside the grid)
      for (int r = tid; r < ni * nj; r += G2P_TILE_THREADS) {
        const int bj = r % nj, bi = r / nj;
        const int gi = oi + bi, gj = oj + bj;
        float *drow = dst + r * nk;
        if (gi < 0 || gi >= snx || gj < 0 || gj >= sny) {
#pragma unroll 4
          for (int bk = 0; bk < nk; ++bk) drow[bk] = 0.f;
          continue;
        }
        const int64_t row = ((int64_t)gi * sny + gj) * snz;
#pragma unroll 4
        for (int bk = 0; bk < nk; ++bk) {
          const int gk = ok + bk;
          drow[bk] = gk >= 0 && gk < snz && GF_IN(row + gk, (int64_t)snx * sny * snz)
                         ? __ldg(src[q] + row + gk)
                         : 0.f;
        }
      }
    }
  }
  if (tx) {  // every thread observes the completed phase (bounded wait)
    long long spins = 0;
    while (!mbar_try_wait(&s_bar, 0)) {
      if (++spins > G2P_WAIT_LIMIT) {
        s_ok = 0;
        break;
      }
    }
  }
  __syncthreads();
  if (!s_ok) {  // record it, give the copies in flight a second bounded wait, leave
    if (tid == 0) {
      atomicAdd(ta.wait_err, 1);
      for (long long k = 0; k < G2P_WAIT_LIMIT && !mbar_try_wait(&s_bar, 0); ++k) {
      }
    }
    __syncthreads();
    return;
  }

  BoxAt bx[6];
#pragma unroll
  for (int q = 0; q < NARR; ++q) {
    const int c = q % 3;
    bx[q] = BoxAt{s_box + (q / 3) * SET + gbox_off(c, KT), I0 - (c != 0), J0 - (c != 1),
                  c == 2 ? K0 : K0 - 4, gbox_nj(c), gbox_nk(c, KT), gbox_vol(c, KT)};
  }
  const float dx = a.dx;
  const int lane = tid & 31, warp = tid >> 5;
  float *const ws = s_out + warp * PW;  // this warp's staging
  int *const wpid = reinterpret_cast<int *>(ws + (APIC ? 480 : 192));
  // per-launch constants: 3 / dx^2 of the C rows (one IEEE division), the clamp margin
  const float inv = __fdiv_rn(3.0f, dx * dx), eps = dx * 1.001f;
  for (int64_t base = b; base < e; base += G2P_TILE_THREADS) {
    const int m = (int)(e - base < G2P_TILE_THREADS ? e - base : G2P_TILE_THREADS);
    if (tid < m) {
      const int64_t q = base + tid;
      const float4 r0 = a.rec0[q];
      const float px = r0.x, py = r0.y, pz = r0.z;
      float gx = div_dx(px, dx, a.inv_dx_exact), gy = div_dx(py, dx, a.inv_dx_exact),
            gz = div_dx(pz, dx, a.inv_dx_exact);
      float hx = gx - 0.5f, hy = gy - 0.5f, hz = gz - 0.5f;
      float nu, nv, nw;
      if (APIC) {
        float c[9];
        const float fxs[3] = {gx, hx, hx}, fys[3] = {hy, gy, hy}, fzs[3] = {hz, hz, gz};
        float vel3[3];
        // the common case: every corner inside the grid and the staged box
        // (the paired gathers); otherwise the clamped gathers of k_g2p
        GStencil gs[3];
        bool lin[3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int snx = nx + (cc == 0), sny = ny + (cc == 1), snz = nz + (cc == 2);
          // stencil_inside, keeping the floors as floats for the gathers
          const float flx = floorf(fxs[cc]), fly = floorf(fys[cc]), flz = floorf(fzs[cc]);
          const int i0 = __float2int_rz(flx), j0 = __float2int_rz(fly), k0 = __float2int_rz(flz);
          const bool inside = i0 >= 0 && i0 < snx - 1 && j0 >= 0 && j0 < sny - 1 && k0 >= 0 &&
                              k0 < snz - 1;
          const int NJ = gbox_nj(cc), NK = gbox_nk(cc, KT);
          lin[cc] = inside && in_box(bx[cc], gbox_ni(cc), i0, i0 + 1, j0, j0 + 1, k0, k0 + 1);
          gs[cc] = GStencil{bx[cc].s + ((i0 - bx[cc].oi) * NJ + (j0 - bx[cc].oj)) * NK +
                                (k0 - bx[cc].ok),
                            NJ * NK, NK, i0, j0, k0, fxs[cc], fys[cc], fzs[cc], flx, fly, flz};
        }
        auto gather_one = [&](int cc) {
          const int snx = nx + (cc == 0), sny = ny + (cc == 1), snz = nz + (cc == 2);
          auto cl = [](int v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); };
          const int i0 = gs[cc].i0, j0 = gs[cc].j0, k0 = gs[cc].k0;
          if (lin[cc])
            apic_gather_lin(gs[cc].p, gs[cc].si, gs[cc].sj, i0, j0, k0, px, py, pz, dx,
                            fxs[cc], fys[cc], fzs[cc], cc, inv, vel3[cc], c[3 * cc],
                            c[3 * cc + 1], c[3 * cc + 2]);
          else if (in_box(bx[cc], gbox_ni(cc), cl(i0, snx), cl(i0 + 1, snx), cl(j0, sny),
                          cl(j0 + 1, sny), cl(k0, snz), cl(k0 + 1, snz)))
            apic_gather_at(bx[cc], px, py, pz, dx, fxs[cc], fys[cc], fzs[cc], snx, sny, snz, cc,
                           inv, vel3[cc], c[3 * cc], c[3 * cc + 1], c[3 * cc + 2]);
          else
            apic_gather(cc == 0 ? a.u : (cc == 1 ? a.v : a.w), px, py, pz, dx, fxs[cc], fys[cc],
                        fzs[cc], snx, sny, snz, cc, inv, vel3[cc], c[3 * cc], c[3 * cc + 1],
                        c[3 * cc + 2]);
        };
        if (lin[0] && lin[1]) {
          float2 v2, c0, c1, c2;
          apic_gather_lin_pair<0, 1>(gs[0], gs[1], px, py, pz, dx, inv, a.one, v2, c0, c1,
                                     c2);
          vel3[0] = v2.x;
          vel3[1] = v2.y;
          c[0] = c0.x, c[1] = c1.x, c[2] = c2.x;
          c[3] = c0.y, c[4] = c1.y, c[5] = c2.y;
        } else {
          gather_one(0);
          gather_one(1);
        }
        if (lin[2])
          apic_gather_lin_k2<2>(gs[2], px, py, pz, dx, inv, a.one, vel3[2], c[6], c[7], c[8]);
        else
          gather_one(2);
        nu = vel3[0];
        nv = vel3[1];
        nw = vel3[2];
#pragma unroll
        for (int k = 0; k < 9; ++k) ws[192 + 9 * lane + k] = c[k];
      } else {
        const float4 r1 = a.rec1[q];
        float pic[3], old[3];
        const float fxs[3] = {gx, hx, hx}, fys[3] = {hy, gy, hy}, fzs[3] = {hz, hz, gz};
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) {
          const int snx = nx + (cc == 0), sny = ny + (cc == 1), snz = nz + (cc == 2);
          float fx = fxs[cc], fy = fys[cc], fz = fzs[cc];
          int i0, j0, k0, i1, j1, k1;
          sample3_index(fx, fy, fz, snx, sny, snz, i0, j0, k0, i1, j1, k1);
          const int NJ = gbox_nj(cc), NK = gbox_nk(cc, KT);
          if (i1 == i0 + 1 && j1 == j0 + 1 && k1 == k0 + 1 &&
              in_box(bx[cc], gbox_ni(cc), i0, i1, j0, j1, k0, k1)) {
            const int off = ((i0 - bx[cc].oi) * NJ + (j0 - bx[cc].oj)) * NK + (k0 - bx[cc].ok);
            const float2 po = sample3_lin_pair(bx[cc].s + off, bx[cc + 3].s + off, NJ * NK, NK,
                                               fx, fy, fz, i0, j0, k0, a.one);
            pic[cc] = po.x;
            old[cc] = po.y;
          } else if (in_box(bx[cc], gbox_ni(cc), i0, i1, j0, j1, k0, k1)) {
            pic[cc] = sample3_at(bx[cc], fx, fy, fz, i0, j0, k0, i1, j1, k1);
            old[cc] = sample3_at(bx[cc + 3], fx, fy, fz, i0, j0, k0, i1, j1, k1);
          } else {
            const float *fp = cc == 0 ? a.u : (cc == 1 ? a.v : a.w);
            const float *fs = cc == 0 ? a.us : (cc == 1 ? a.vs : a.ws);
            const int64_t nf = (int64_t)snx * sny * snz;
            pic[cc] = sample3_at(GlobalAt{fp, (int64_t)sny * snz, snz, nf}, fx, fy, fz, i0, j0,
                                 k0, i1, j1, k1);
            old[cc] = sample3_at(GlobalAt{fs, (int64_t)sny * snz, snz, nf}, fx, fy, fz, i0, j0,
                                 k0, i1, j1, k1);
          }
        }
        float fu = r1.x + (pic[0] - old[0]), fv = r1.y + (pic[1] - old[1]),
              fw = r1.z + (pic[2] - old[2]);
        float ob = 1.0f - a.flip_blend;
        nu = a.flip_blend * fu + ob * pic[0];
        nv = a.flip_blend * fv + ob * pic[1];
        nw = a.flip_blend * fw + ob * pic[2];
      }
      ws[96 + 3 * lane] = nu;
      ws[96 + 3 * lane + 1] = nv;
      ws[96 + 3 * lane + 2] = nw;
      ws[3 * lane] = clampf(px + nu * a.dt, eps, a.dom0 - eps);
      ws[3 * lane + 1] = clampf(py + nv * a.dt, eps, a.dom1 - eps);
      ws[3 * lane + 2] = clampf(pz + nw * a.dt, eps, a.dom2 - eps);
      wpid[lane] = __float_as_int(r0.w);
    }
    // the warp writes its particles' outputs: each store instruction covers
    // 32 consecutive floats of one array (whole 128-byte spans)
    __syncwarp();
    const int mw = m - warp * 32 < 0 ? 0 : (m - warp * 32 > 32 ? 32 : m - warp * 32);
    const int64_t wb = base + warp * 32;
    float *const gp = a.pos + 3 * wb, *const gv = a.vel + 3 * wb;
    if (mw == 32) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        gp[lane + 32 * k] = ws[lane + 32 * k];
        gv[lane + 32 * k] = ws[96 + lane + 32 * k];
      }
      if (APIC) {
        float *const gc = a.C + 9 * wb;
#pragma unroll
        for (int k = 0; k < 9; ++k) gc[lane + 32 * k] = ws[192 + lane + 32 * k];
      }
      a.pid[wb + lane] = wpid[lane];
    } else if (mw > 0) {
      for (int k = lane; k < 3 * mw; k += 32) {
        gp[k] = ws[k];
        gv[k] = ws[96 + k];
      }
      if (APIC)
        for (int k = lane; k < 9 * mw; k += 32) a.C[9 * wb + k] = ws[192 + k];
      if (lane < mw) a.pid[wb + lane] = wpid[lane];
    }
    __syncwarp();
  }
}

// Tensor maps of the bound face arrays for k_g2p_tile (single-grid contexts).
// cuTensorMapEncodeTiled is reached through the runtime's driver entry point,
// so the library does not link the driver library directly.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

int encode_face_maps(Ctx *c) {
  FaceMaps *sets[2] = {&c->face_maps, &c->face_maps2};
  for (FaceMaps *fm : sets) fm->mask = 0;
  if (c->nseg > 0) return GF_OK;  // batches use the per-particle G2P
  EncodeTiledFn fn = encode_fn();
  if (!fn) return GF_OK;  // plain loads for every box
  const float *arr[6] = {c->f.u, c->f.v, c->f.w, c->f.us, c->f.vs, c->f.ws};
  for (int kt = 1; kt <= 2; ++kt) {
    FaceMaps *fm = sets[kt - 1];
    for (int q = 0; q < 6; ++q) {
      const int comp = q % 3;
      const uint64_t snx = c->nx + (comp == 0), sny = c->ny + (comp == 1),
                     snz = c->nz + (comp == 2);
      const cuuint64_t dims[3] = {snz, sny, snx};
      const cuuint64_t strides[2] = {snz * 4, sny * snz * 4};
      const cuuint32_t box[3] = {(cuuint32_t)gbox_nk(comp, kt), (cuuint32_t)gbox_nj(comp),
                                 (cuuint32_t)gbox_ni(comp)};
      const cuuint32_t estr[3] = {1, 1, 1};
      if (reinterpret_cast<uintptr_t>(arr[q]) % 16 || strides[0] % 16 || strides[1] % 16)
        continue;
      if (fn(&fm->m[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(arr[q]), dims,
             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        fm->mask |= 1 << q;
    }
  }
  return GF_OK;
}

// ------------------------------------------------------------- batches
// The stage kernels over a batch of scenes: every item (tile, face slot,
// cell, particle) finds its scene in the segment table and runs the
// single-grid body on that scene's view of the concatenated arrays.
struct BatchArgs {
  SegIndex sx;
  const int32_t *start;
  const float4 *rec0, *rec1, *rec2, *rec3;
  float *u, *v, *w, *uw, *vw, *ww, *us, *vs, *ws;
  const uint8_t *label;
  float *div;
  const float *p;
  float *pos, *vel, *C;
  int32_t *pid;
  int64_t n;
  float dt, flip_blend, rho;
};

__device__ __forceinline__ GridArgs grid_view(const BatchArgs &b, const SegRow &r) {
  GridArgs a;
  a.u = b.u + r.fu0; a.v = b.v + r.fv0; a.w = b.w + r.fw0;
  a.us = b.us + r.fu0; a.vs = b.vs + r.fv0; a.ws = b.ws + r.fw0;
  a.uw = b.uw + r.fu0; a.vw = b.vw + r.fv0; a.ww = b.ww + r.fw0;
  a.label = b.label + r.cell0;
  a.solid_u = a.solid_v = a.solid_w = nullptr;  // static solids in a batch
  a.div = b.div + r.cell0;
  a.p = b.p + r.cell0;
  a.nx = r.nx; a.ny = r.ny; a.nz = r.nz;
  return a;
}

template <bool APIC, int MAP>
__global__ void __launch_bounds__(256, MAP >= 2 ? GF_P2G_MINB : 1) kb_p2g_tile(BatchArgs b) {
  const int64_t t = blockIdx.x;
  const int s = seg_find(b.sx.tile0, b.sx.n, t);
  const SegRow r = b.sx.row[s];
  P2GArgs a{b.start, b.rec0, b.rec1, b.rec2, b.rec3, b.u + r.fu0, b.v + r.fv0, b.w + r.fw0,
            b.uw + r.fu0, b.vw + r.fv0, b.ww + r.fw0, r.dx, r.nx, r.ny, r.nz, r.nty, r.ntz,
            exact_inverse(r.dx)};
  p2g_tile_body<APIC, 1, MAP>(a, (int)(t - r.tile0), t * TILE_CELLS, 1);
}

__global__ void kb_forces(BatchArgs b, int64_t nslot, float gravity) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nslot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int s = seg_find(b.sx.fslot0, b.sx.n, q);
    const SegRow r = b.sx.row[s];
    const float gd = gravity * b.dt;
    forces_slot(grid_view(b, r), q - r.fslot0, gd);
  }
}

__global__ void kb_divergence(BatchArgs b, int64_t ncell) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int s = seg_find(b.sx.cell0, b.sx.n, c);
    const SegRow r = b.sx.row[s];
    float scale = b.rho * r.dx;  // (rho * dx) / dt per scene
    scale = scale / b.dt;
    divergence_cell(grid_view(b, r), c - r.cell0, scale);
  }
}

__global__ void kb_project(BatchArgs b, int64_t nslot) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nslot;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int s = seg_find(b.sx.fslot0, b.sx.n, q);
    const SegRow r = b.sx.row[s];
    float scale = b.rho * r.dx;  // dt / (rho * dx) per scene
    scale = b.dt / scale;
    project_slot(grid_view(b, r), q - r.fslot0, scale);
  }
}

template <bool APIC>
__global__ void __launch_bounds__(512) kb_g2p(BatchArgs b) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= b.n) return;
  const int s = seg_find(b.sx.part0, b.sx.n, q);
  const SegRow r = b.sx.row[s];
  G2PArgs a{b.rec0, b.rec1, b.u + r.fu0, b.v + r.fv0, b.w + r.fw0, b.us + r.fu0,
            b.vs + r.fv0, b.ws + r.fw0, b.pos, b.vel, b.C, b.pid, b.n, r.dx, b.dt,
            b.flip_blend, r.dom0, r.dom1, r.dom2, r.nx, r.ny, r.nz, exact_inverse(r.dx)};
  g2p_particle<APIC>(a, q);
}

static BatchArgs batch_args(Ctx *c) {
  BatchArgs b{};
  b.sx = seg_index(c);
  b.start = c->start;
  b.rec0 = c->rec0; b.rec1 = c->rec1; b.rec2 = c->rec2; b.rec3 = c->rec3;
  b.u = c->f.u; b.v = c->f.v; b.w = c->f.w;
  b.uw = c->f.uw; b.vw = c->f.vw; b.ww = c->f.ww;
  b.us = c->f.us; b.vs = c->f.vs; b.ws = c->f.ws;
  b.label = c->f.label; b.div = c->f.div; b.p = c->f.p;
  b.pos = c->p.pos; b.vel = c->p.vel; b.C = c->p.C; b.pid = c->p.pid;
  b.n = c->p.n;
  return b;
}

// ------------------------------------------------------------------- CFL
__global__ void k_vmax(const float *__restrict__ vel, int64_t n, float *out) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float x = vel[3 * i], y = vel[3 * i + 1], z = vel[3 * i + 2];
    float s = x * x + y * y + z * z;
    m = fmaxf(m, s);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out), __float_as_int(m));
}

// ------------------------------------------------------------- launchers
static inline unsigned grid_for(int64_t n, int threads, int num_sms) {
  int64_t g = (n + threads - 1) / threads;
  int64_t cap = (int64_t)num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

// Zero the six face arrays P2G accumulates into, in one launch (six memsets
// cost six graph nodes): each array's 16-byte-aligned body with 16-byte
// stores, its unaligned head and tail with 4-byte stores.
struct ZeroFaces {
  float *p[6];
  int64_t n[6];
};
__global__ void k_zero_faces(ZeroFaces z) {
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    float *const p = z.p[q];
    const int64_t n = z.n[q];
    int64_t head = (int64_t)(((16u - (uint32_t)(reinterpret_cast<uintptr_t>(p) & 15u)) & 15u) >> 2);
    if (head > n) head = n;
    const int64_t nv = (n - head) >> 2;
    float4 *const v = reinterpret_cast<float4 *>(p + head);
    for (int64_t i = t0; i < nv; i += stride) v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t0 < head) p[t0] = 0.f;
    for (int64_t i = head + 4 * nv + t0; i < n; i += stride) p[i] = 0.f;
  }
}

int launch_p2g(Ctx *c, int transfer) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_p2g: buffers not bound");
  if (transfer == GF_APIC && !c->p.C) return fail(c, GF_INVALID_ARG, "gf_p2g: APIC needs C");
  cudaStream_t st = c->stream;
  {
    const ZeroFaces z{{c->f.u, c->f.uw, c->f.v, c->f.vw, c->f.w, c->f.ww},
                      {c->nu, c->nu, c->nv, c->nv, c->nw, c->nw}};
    k_zero_faces<<<(unsigned)((c->num_sms > 0 ? c->num_sms : 148) * 4), 512, 0, st>>>(z);
    c->launches++;
  }
  P2GArgs a{c->start, c->rec0, c->rec1, c->rec2, c->rec3, c->f.u, c->f.v, c->f.w,
            c->f.uw, c->f.vw, c->f.ww, c->dx, c->nx, c->ny, c->nz, c->nty, c->ntz,
            exact_inverse(c->dx)};
  if (c->p.n > 0 && c->nseg > 0) {
    BatchArgs b = batch_args(c);
    const int map = c->tune.p2g_map;
    const size_t sm = p2g_smem_bytes(1, map, transfer == GF_APIC);
    auto launch = [&](auto kern) {
      if (sm > 48 * 1024)
        cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
      kern<<<c->ntiles, 256, sm, st>>>(b);
    };
    if (transfer == GF_APIC) {
      if (map == 5) launch(kb_p2g_tile<true, 5>);
      else if (map == 4) launch(kb_p2g_tile<true, 4>);
      else if (map == 3) launch(kb_p2g_tile<true, 3>);
      else if (map == 2) kb_p2g_tile<true, 2><<<c->ntiles, 256, sm, st>>>(b);
      else if (map == 1) kb_p2g_tile<true, 1><<<c->ntiles, 256, sm, st>>>(b);
      else kb_p2g_tile<true, 0><<<c->ntiles, 256, sm, st>>>(b);
    } else {
      if (map == 5) launch(kb_p2g_tile<false, 5>);
      else if (map == 4) launch(kb_p2g_tile<false, 4>);
      else if (map == 3) launch(kb_p2g_tile<false, 3>);
      else if (map == 2) kb_p2g_tile<false, 2><<<c->ntiles, 256, sm, st>>>(b);
      else if (map == 1) kb_p2g_tile<false, 1><<<c->ntiles, 256, sm, st>>>(b);
      else kb_p2g_tile<false, 0><<<c->ntiles, 256, sm, st>>>(b);
    }
    c->launches++;
  } else if (c->p.n > 0) {
    const int kt = c->tune.p2g_tiles_k == 2 ? 2 : 1;
    const unsigned g = (unsigned)(c->ntx * c->nty * ((c->ntz + kt - 1) / kt));
    const int map = c->tune.p2g_map >= 0 && c->tune.p2g_map <= 5 ? c->tune.p2g_map : 0;
    const size_t sm = p2g_smem_bytes(kt, map, transfer == GF_APIC);
    auto launch = [&](auto kern) {
      if (sm > 48 * 1024)
        cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
      kern<<<g, 256, sm, st>>>(a);
    };
    if (transfer == GF_APIC) {
      if (map == 5) kt == 2 ? launch(k_p2g_tile<true, 2, 5>) : launch(k_p2g_tile<true, 1, 5>);
      else if (map == 4) kt == 2 ? launch(k_p2g_tile<true, 2, 4>) : launch(k_p2g_tile<true, 1, 4>);
      else if (map == 3) kt == 2 ? launch(k_p2g_tile<true, 2, 3>) : launch(k_p2g_tile<true, 1, 3>);
      else if (map == 2) kt == 2 ? launch(k_p2g_tile<true, 2, 2>) : launch(k_p2g_tile<true, 1, 2>);
      else if (map) kt == 2 ? launch(k_p2g_tile<true, 2, 1>) : launch(k_p2g_tile<true, 1, 1>);
      else     kt == 2 ? launch(k_p2g_tile<true, 2, 0>) : launch(k_p2g_tile<true, 1, 0>);
    } else {
      if (map == 5) kt == 2 ? launch(k_p2g_tile<false, 2, 5>) : launch(k_p2g_tile<false, 1, 5>);
      else if (map == 4) kt == 2 ? launch(k_p2g_tile<false, 2, 4>) : launch(k_p2g_tile<false, 1, 4>);
      else if (map == 3) kt == 2 ? launch(k_p2g_tile<false, 2, 3>) : launch(k_p2g_tile<false, 1, 3>);
      else if (map == 2) kt == 2 ? launch(k_p2g_tile<false, 2, 2>) : launch(k_p2g_tile<false, 1, 2>);
      else if (map) kt == 2 ? launch(k_p2g_tile<false, 2, 1>) : launch(k_p2g_tile<false, 1, 1>);
      else     kt == 2 ? launch(k_p2g_tile<false, 2, 0>) : launch(k_p2g_tile<false, 1, 0>);
    }
    c->launches++;
  }
  return check_launch(c, "gf_p2g");
}

static GridArgs grid_args(Ctx *c) {
  GridArgs a;
  a.u = c->f.u; a.v = c->f.v; a.w = c->f.w;
  a.us = c->f.us; a.vs = c->f.vs; a.ws = c->f.ws;
  a.uw = c->f.uw; a.vw = c->f.vw; a.ww = c->f.ww;
  a.label = c->f.label;
  a.solid_u = c->f.solid_u; a.solid_v = c->f.solid_v; a.solid_w = c->f.solid_w;
  a.div = c->f.div; a.p = c->f.p;
  a.nx = c->nx; a.ny = c->ny; a.nz = c->nz;
  return a;
}

static inline unsigned grid_tuned(const Ctx *c, int64_t n) {
  int64_t g = (n + c->tune.grid_threads - 1) / c->tune.grid_threads;
  int64_t cap = (int64_t)c->num_sms * c->tune.grid_blocks_per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

int launch_forces_div(Ctx *c, float gravity, float dt, float rho) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_forces_div: buffers not bound");
  if (c->nseg > 0) {
    BatchArgs b = batch_args(c);
    b.dt = dt;
    b.rho = rho;
    const int th = c->tune.grid_threads;
    kb_forces<<<grid_tuned(c, c->nfslot), th, 0, c->stream>>>(b, c->nfslot, gravity);
    kb_divergence<<<grid_tuned(c, c->ncell), th, 0, c->stream>>>(b, c->ncell);
    c->launches += 2;
    return check_launch(c, "gf_forces_div");
  }
  GridArgs a = grid_args(c);
  float gd = gravity * dt;        // g * dt in float32, as k3_add_gravity
  float scale = rho * c->dx;      // (rho * dx) / dt, as k3_compute_divergence
  scale = scale / dt;
  const int th = c->tune.grid_threads;
  k_forces<<<grid_tuned(c, c->nfslot), th, 0, c->stream>>>(a, gd);
  k_divergence<<<grid_tuned(c, c->ncell), th, 0, c->stream>>>(a, scale);
  c->launches += 2;
  return check_launch(c, "gf_forces_div");
}

int launch_project(Ctx *c, float dt, float rho) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_project: buffers not bound");
  const int th = c->tune.grid_threads;
  if (c->nseg > 0) {
    BatchArgs b = batch_args(c);
    b.dt = dt;
    b.rho = rho;
    kb_project<<<grid_tuned(c, c->nfslot), th, 0, c->stream>>>(b, c->nfslot);
    c->launches++;
    return check_launch(c, "gf_project");
  }
  GridArgs a = grid_args(c);
  float scale = rho * c->dx;  // dt / (rho * dx), as k3_subtract_pressure_grad
  scale = dt / scale;
  k_project<<<grid_tuned(c, c->nfslot), th, 0, c->stream>>>(a, scale);
  c->launches++;
  return check_launch(c, "gf_project");
}

int launch_g2p(Ctx *c, int transfer, float flip_blend, float dt) {
  if (!c->bound) return fail(c, GF_INVALID_ARG, "gf_g2p: buffers not bound");
  if (transfer == GF_APIC && !c->p.C) return fail(c, GF_INVALID_ARG, "gf_g2p: APIC needs C");
  if (c->p.n == 0) return GF_OK;
  const int th = c->tune.g2p_threads;
  const unsigned g = (unsigned)((c->p.n + th - 1) / th);
  if (c->nseg > 0) {
    BatchArgs b = batch_args(c);
    b.dt = dt;
    b.flip_blend = flip_blend;
    if (transfer == GF_APIC)
      kb_g2p<true><<<g, th, 0, c->stream>>>(b);
    else
      kb_g2p<false><<<g, th, 0, c->stream>>>(b);
    c->launches++;
    return check_launch(c, "gf_g2p");
  }
  G2PArgs a{c->rec0, c->rec1, c->f.u, c->f.v, c->f.w, c->f.us, c->f.vs, c->f.ws,
            c->p.pos, c->p.vel, c->p.C, c->p.pid, c->p.n, c->dx, dt, flip_blend,
            c->dom[0], c->dom[1], c->dom[2], c->nx, c->ny, c->nz, exact_inverse(c->dx)};
  if (c->tune.g2p_tiles_k == 0) {  // no staging: one thread per particle, L1/L2 gathers
    if (transfer == GF_APIC)
      k_g2p<true><<<g, th, 0, c->stream>>>(a);
    else
      k_g2p<false><<<g, th, 0, c->stream>>>(a);
    c->launches++;
    return check_launch(c, "gf_g2p");
  }
  G2PTileArgs ta{a, c->start, c->nty, c->ntz, c->health + 5};
  const int kt = c->tune.g2p_tiles_k == 2 ? 2 : 1;
  const unsigned gb =
      (unsigned)(c->ntx * c->nty * ((c->ntz + kt - 1) / kt) * G2P_SPLITS * kt);
  const FaceMaps &fm = kt == 2 ? c->face_maps2 : c->face_maps;
  auto launch = [&](auto kern, int mode) {
    const size_t sm = g2p_smem_bytes(mode, kt);  // beside the static staging buffers
    cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    kern<<<gb, G2P_TILE_THREADS, sm, c->stream>>>(ta, fm);
  };
  if (transfer == GF_APIC)
    kt == 2 ? launch(k_g2p_tile<GF_APIC, 2>, GF_APIC) : launch(k_g2p_tile<GF_APIC, 1>, GF_APIC);
  else
    kt == 2 ? launch(k_g2p_tile<GF_FLIP, 2>, GF_FLIP) : launch(k_g2p_tile<GF_FLIP, 1>, GF_FLIP);
  c->launches++;
  return check_launch(c, "gf_g2p");
}

int launch_vmax(Ctx *c) {
  int e = check_cuda(c, cudaMemsetAsync(c->vmax_dev, 0, 4, c->stream), "memset vmax");
  if (e) return e;
  if (c->p.n > 0) {
    k_vmax<<<grid_for(c->p.n, 256, c->num_sms), 256, 0, c->stream>>>(c->p.vel, c->p.n,
                                                                     c->vmax_dev);
    c->launches++;
  }
  return check_launch(c, "gf_vmax");
}

GF_BOUNDS_READER(transfer)

}  // namespace gf
