// Adjoint of one PIC substep, with the cell labels held fixed.
//
// Forward map of a substep (particles in the sorted order of its binning):
//   P2G      m_f = sum_p W_pf(x_p),  q_f = sum_p W_pf v_p,c(f)        (k3_p2g)
//   normalize u_f = q_f / m_f  (m_f > 1e-8, else 0)                 (k3_normalize)
//   forces   v faces += g dt; boundary faces <- 0                  (k3_add_gravity, bc)
//   project  p = A^-1(-div(u)),  u3 = bc(u - k grad p)              (:846-871, PCG, :1364-1407)
//   G2P      v'_p = sum_f S_pf(x_p) u3_f                           (k3_g2p_and_advect, blend 0)
//   advect   x'_p = clamp(x_p + v'_p dt)
// Adjoint (this file), given xbar', vbar' of the outputs:
//   k_adj_g2p    vbar'' = vbar' + dt xbar' (unclamped axes), xbar = xbar' (unclamped);
//                ubar3_f += S_pf vbar''  (scatter), xbar += dS/dx . u3 vbar''
//   k_adj_grad   pbar_c = sum over c's faces of -/+ k ubar3_f   (pressure-gradient adjoint)
//   (solve)      A lambda = pbar  -> divbar = -lambda  (same SPD operator, gf_pressure)
//   k_adj_faces  ubar = bc ? 0 : ubar3 + s (divbar_left - divbar_right);
//                qbar = ubar / m,  mbar = -ubar u / m
//   k_adj_p2g    vbar_p += sum_f W_pf qbar_f (gather), xbar_p += dW/dx (v qbar + mbar)
// Weight derivatives: W = wx wy wz, wx = 1 - sx or sx, sx = x/dx - offset - i0,
// so dW/dx = (-1 or +1) / dx * wy wz (and likewise for y, z).
#include "gf_internal.cuh"

namespace gf {

struct AdjArgs {
  // sorted inputs of the substep: (x,y,z,pid), then FLIP/PIC (vx,vy,vz,-),
  // APIC one record per component c: (v_c, C row c) in rec1, rec2, rec3
  const float4 *rec0, *rec1;
  const float4 *rec2, *rec3;
  const float *Cbar_out;      // APIC: (n,9) adjoint of the output C, sorted order
  float *Cbar_in;             // APIC: (n,9) adjoint of the input C, storage order
  const int32_t *order;       // storage slot (input order) of each sorted position
  const float *m[3];          // P2G weight sums per component
  const float *un[3];         // normalised P2G velocities (pre-force)
  const float *u3[3];         // final face velocities
  const uint8_t *label;
  float *ubar3[3], *qbar[3], *mbar[3];
  float *div_io;              // pbar in, then -lambda read back as divbar
  const float *lambda;        // adjoint pressure solution
  const float *xbar_out, *vbar_out;  // (n,3), sorted order of this substep
  float *xbar_acc;            // (n,3) scratch
  float *xbar_in, *vbar_in;   // (n,3), input storage order
  int64_t n;
  float dx, dt, rho, dom0, dom1, dom2;
  int nx, ny, nz;
};

__device__ __forceinline__ float clampf_(float x, float lo, float hi) {
  return x < lo ? lo : (x > hi ? hi : x);
}

// sample3 weights of gridmath.py:29-63 for one component: corner indices,
// weights and, per axis, d(weight)/dx scale (0 when the coordinate is clamped).
struct Corners {
  int64_t idx[8];
  float w[8];
  float dw[8][3];
};

__device__ __forceinline__ void sample_corners(float fx, float fy, float fz, int nxm, int nym,
                                               int nzm, float inv_dx, Corners &c) {
  const bool cx = fx < 0.0f || fx > (float)nxm, cy = fy < 0.0f || fy > (float)nym,
             cz = fz < 0.0f || fz > (float)nzm;
  fx = clampf_(fx, 0.0f, (float)nxm);
  fy = clampf_(fy, 0.0f, (float)nym);
  fz = clampf_(fz, 0.0f, (float)nzm);
  int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
      k0 = __float2int_rz(floorf(fz));
  if (i0 >= nxm) i0 = nxm - 1;
  if (j0 >= nym) j0 = nym - 1;
  if (k0 >= nzm) k0 = nzm - 1;
  if (i0 < 0) i0 = 0;
  if (j0 < 0) j0 = 0;
  if (k0 < 0) k0 = 0;
  int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  if (i1 >= nxm) i1 = nxm - 1;
  if (j1 >= nym) j1 = nym - 1;
  if (k1 >= nzm) k1 = nzm - 1;
  const float rsx = fx - (float)i0, rsy = fy - (float)j0, rsz = fz - (float)k0;
  const float sx = clampf_(rsx, 0.0f, 1.0f), sy = clampf_(rsy, 0.0f, 1.0f),
              sz = clampf_(rsz, 0.0f, 1.0f);
  const float gx = (cx || rsx < 0.0f || rsx > 1.0f) ? 0.0f : inv_dx;
  const float gy = (cy || rsy < 0.0f || rsy > 1.0f) ? 0.0f : inv_dx;
  const float gz = (cz || rsz < 0.0f || rsz > 1.0f) ? 0.0f : inv_dx;
  const int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
  const float sgn[2] = {-1.0f, 1.0f};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int q = (a * 2 + b) * 2 + e;
        c.idx[q] = ((int64_t)ii[a] * nym + jj[b]) * nzm + kk[e];
        c.w[q] = wx[a] * wy[b] * wz[e];
        c.dw[q][0] = sgn[a] * gx * wy[b] * wz[e];
        c.dw[q][1] = sgn[b] * gy * wx[a] * wz[e];
        c.dw[q][2] = sgn[e] * gz * wx[a] * wy[b];
      }
}

// scatter_face weights of gridmath.py:70-95 (P2G): corners dropped when out of
// the component's grid; idx = -1 for a dropped corner.
__device__ __forceinline__ void scatter_corners(float fx, float fy, float fz, int snx, int sny,
                                                int snz, float inv_dx, Corners &c) {
  const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
            k0 = __float2int_rz(floorf(fz));
  const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
  const float sgn[2] = {-1.0f, 1.0f};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int q = (a * 2 + b) * 2 + e;
        const int ii = i0 + a, jj = j0 + b, kk = k0 + e;
        const bool in = ii >= 0 && ii < snx && jj >= 0 && jj < sny && kk >= 0 && kk < snz;
        c.idx[q] = in ? ((int64_t)ii * sny + jj) * snz + kk : -1;
        c.w[q] = wx[a] * wy[b] * wz[e];
        c.dw[q][0] = sgn[a] * inv_dx * wy[b] * wz[e];
        c.dw[q][1] = sgn[b] * inv_dx * wx[a] * wz[e];
        c.dw[q][2] = sgn[e] * inv_dx * wx[a] * wy[b];
      }
}

__device__ __forceinline__ void adj_g2p_item(const AdjArgs &a, int64_t q) {
  const float4 r0 = a.rec0[q];
  const float p[3] = {r0.x, r0.y, r0.z};
  const float inv_dx = 1.0f / a.dx;
  const float g[3] = {__fdiv_rn(p[0], a.dx), __fdiv_rn(p[1], a.dx), __fdiv_rn(p[2], a.dx)};
  const float h[3] = {g[0] - 0.5f, g[1] - 0.5f, g[2] - 0.5f};
  const int sz[3][3] = {{a.nx + 1, a.ny, a.nz}, {a.nx, a.ny + 1, a.nz}, {a.nx, a.ny, a.nz + 1}};
  const float dom[3] = {a.dom0, a.dom1, a.dom2};
  const float eps = a.dx * 1.001f;
  Corners cs[3];
  float vnew[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    sample_corners(c == 0 ? g[0] : h[0], c == 1 ? g[1] : h[1], c == 2 ? g[2] : h[2], sz[c][0],
                   sz[c][1], sz[c][2], inv_dx, cs[c]);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += cs[c].w[k] * a.u3[c][cs[c].idx[k]];
    vnew[c] = acc;
  }
  float xb[3], vb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float xo = a.xbar_out[3 * q + d], vo = a.vbar_out[3 * q + d];
    const float xn = p[d] + vnew[d] * a.dt;
    const bool free = xn >= eps && xn <= dom[d] - eps;
    xb[d] = free ? xo : 0.0f;
    vb[d] = vo + (free ? a.dt * xo : 0.0f);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float uv = a.u3[c][cs[c].idx[k]];
      atomicAdd(&a.ubar3[c][cs[c].idx[k]], cs[c].w[k] * vb[c]);
#pragma unroll
      for (int d = 0; d < 3; ++d) xb[d] += cs[c].dw[k][d] * uv * vb[c];
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) a.xbar_acc[3 * q + d] = xb[d];
}

__global__ void k_adj_g2p(AdjArgs a) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < a.n) adj_g2p_item(a, q);
}

// Gradient step adjoint, per cell: pbar_c = sum_f dU2_f/dp_c * ubar3_f over
// the faces where k3_subtract_pressure_grad acts (both sides non-solid, one
// fluid, interior face); p of a non-fluid cell is a constant 0.
__device__ __forceinline__ void adj_grad_item(const AdjArgs &a, int64_t c, float k) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  {
    if (a.label[c] != 1) {
      a.div_io[c] = 0.0f;
      return;
    }
    const int kk = (int)(c % nz);
    const int64_t rr = c / nz;
    const int j = (int)(rr % ny), i = (int)(rr / ny);
    const int64_t sx = (int64_t)ny * nz;
    float pb = 0.0f;
    // u faces i (c on its right: u -= k (p_c - p_left)) and i+1 (c on its left)
    if (i >= 1) {
      const int ml = a.label[c - sx];
      if (ml != 2) pb -= k * a.ubar3[0][((int64_t)i * ny + j) * nz + kk];
    }
    if (i + 1 <= nx - 1) {
      const int mr = a.label[c + sx];
      if (mr != 2) pb += k * a.ubar3[0][((int64_t)(i + 1) * ny + j) * nz + kk];
    }
    if (j >= 1) {
      const int mb = a.label[c - nz];
      if (mb != 2) pb -= k * a.ubar3[1][((int64_t)i * (ny + 1) + j) * nz + kk];
    }
    if (j + 1 <= ny - 1) {
      const int mt = a.label[c + nz];
      if (mt != 2) pb += k * a.ubar3[1][((int64_t)i * (ny + 1) + j + 1) * nz + kk];
    }
    if (kk >= 1) {
      const int mba = a.label[c - 1];
      if (mba != 2) pb -= k * a.ubar3[2][((int64_t)i * ny + j) * (nz + 1) + kk];
    }
    if (kk + 1 <= nz - 1) {
      const int mfr = a.label[c + 1];
      if (mfr != 2) pb += k * a.ubar3[2][((int64_t)i * ny + j) * (nz + 1) + kk + 1];
    }
    a.div_io[c] = pb;
  }
}

__global__ void k_adj_grad(AdjArgs a, float k) {
  const int64_t n = (int64_t)a.nx * a.ny * a.nz;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    adj_grad_item(a, c, k);
}

// Divergence + boundary + normalisation adjoint, per face.
__device__ __forceinline__ void adj_faces_item(const AdjArgs &a, int64_t t, float s) {
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  {
    const int k = (int)(t % (nz + 1));
    const int64_t rr = t / (nz + 1);
    const int j = (int)(rr % (ny + 1)), i = (int)(rr / (ny + 1));
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
      const int ex = comp == 0, ey = comp == 1, ez = comp == 2;
      if (i > nx - 1 + ex || j > ny - 1 + ey || k > nz - 1 + ez) continue;
      const int sny = ny + ey, snz = nz + ez;
      const int64_t g = ((int64_t)i * sny + j) * snz + k;
      // cells on the low (L) and high (R) side of the face along comp's axis
      const int li = i - ex, lj = j - ey, lk = k - ez;
      const bool hasL = li >= 0 && lj >= 0 && lk >= 0;
      const bool hasR = i < nx && j < ny && k < nz;
      const int64_t cL = hasL ? ((int64_t)li * ny + lj) * nz + lk : 0;
      const int64_t cR = hasR ? ((int64_t)i * ny + j) * nz + k : 0;
      const int mL = hasL ? a.label[cL] : 2, mR = hasR ? a.label[cR] : 2;
      const bool bc = !hasL || !hasR || mL == 2 || mR == 2;  // k3_enforce_solid_bc faces
      float ub = 0.0f;
      if (!bc) {
        ub = a.ubar3[comp][g];
        // div_c = s (sum out - in): this face is L's "out" face, R's "in" face;
        // divbar = -lambda
        if (mL == 1) ub += s * (-a.lambda[cL]);
        if (mR == 1) ub -= s * (-a.lambda[cR]);
      }
      const float m = a.m[comp][g];
      const bool ok = m > 1.0e-8f;
      a.qbar[comp][g] = ok ? ub / m : 0.0f;
      a.mbar[comp][g] = ok ? -ub * a.un[comp][g] / m : 0.0f;
    }
  }
}

__global__ void k_adj_faces(AdjArgs a, float s) {
  const int64_t nf = (int64_t)(a.nx + 1) * (a.ny + 1) * (a.nz + 1);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf;
       t += (int64_t)gridDim.x * blockDim.x)
    adj_faces_item(a, t, s);
}


__device__ __forceinline__ void adj_p2g_item(const AdjArgs &a, int64_t q) {
  const float4 r0 = a.rec0[q], r1 = a.rec1[q];
  const float vel[3] = {r1.x, r1.y, r1.z};
  const float inv_dx = 1.0f / a.dx;
  const float g[3] = {__fdiv_rn(r0.x, a.dx), __fdiv_rn(r0.y, a.dx), __fdiv_rn(r0.z, a.dx)};
  const float h[3] = {g[0] - 0.5f, g[1] - 0.5f, g[2] - 0.5f};
  const int sz[3][3] = {{a.nx + 1, a.ny, a.nz}, {a.nx, a.ny + 1, a.nz}, {a.nx, a.ny, a.nz + 1}};
  float xb[3] = {a.xbar_acc[3 * q], a.xbar_acc[3 * q + 1], a.xbar_acc[3 * q + 2]};
  float vb[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Corners cs;
    scatter_corners(c == 0 ? g[0] : h[0], c == 1 ? g[1] : h[1], c == 2 ? g[2] : h[2], sz[c][0],
                    sz[c][1], sz[c][2], inv_dx, cs);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (cs.idx[k] < 0) continue;
      const float qb = a.qbar[c][cs.idx[k]], mb = a.mbar[c][cs.idx[k]];
      vb[c] += cs.w[k] * qb;
      const float coef = vel[c] * qb + mb;
#pragma unroll
      for (int d = 0; d < 3; ++d) xb[d] += cs.dw[k][d] * coef;
    }
  }
  const int64_t s = a.order[q];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    a.xbar_in[3 * s + d] = xb[d];
    a.vbar_in[3 * s + d] = vb[d];
  }
}

__global__ void k_adj_p2g(AdjArgs a) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < a.n) adj_p2g_item(a, q);
}

// ---- APIC adjoint --------------------------------------------------------
// Forward (k3_p2g_apic :1475-1588, k3_g2p_apic_advect :1591-1732), per
// component c with face offsets o_f = x_f - x_p:
//   P2G   q_f = sum_p W_pf (v_pc + C_p[c] . o_f),  m_f = sum_p W_pf
//   G2P   v'_pc = sum_f S_pf u3_f,  C'_p[c][d] = inv sum_f S_pf u3_f o_fd
//         (S: clamped corner indices, unclamped weights; inv = 3 / dx^2)
// Adjoint: g_f = vb_c + inv (o_f . Cbar'[c]) carries both outputs back,
//   ubar3_f += S_pf g_f;  xbar += dS/dx u3_f g_f - inv (sum_f S_pf u3_f) Cbar'[c]
//   P2G: vbar_c += sum W qbar,  Cbar[c] += sum W qbar o_f,
//        xbar += dW/dx (val qbar + mbar) - (sum W qbar) C[c].

// Corners of the APIC gather: indices clamped into the grid, weights from
// s = f - floor(f) unclamped (so d/df is never gated).
__device__ __forceinline__ void apic_corners(float fx, float fy, float fz, int snx, int sny,
                                             int snz, int ax, float dx, float inv_dx, float px,
                                             float py, float pz, Corners &c, float (&o)[8][3]) {
  const int i0 = __float2int_rz(floorf(fx)), j0 = __float2int_rz(floorf(fy)),
            k0 = __float2int_rz(floorf(fz));
  const float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  const float wx[2] = {1.0f - sx, sx}, wy[2] = {1.0f - sy, sy}, wz[2] = {1.0f - sz, sz};
  const float sgn[2] = {-1.0f, 1.0f};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int q = (a * 2 + b) * 2 + e;
        int ii = i0 + a, jj = j0 + b, kk = k0 + e;
        ii = ii < 0 ? 0 : (ii > snx - 1 ? snx - 1 : ii);
        jj = jj < 0 ? 0 : (jj > sny - 1 ? sny - 1 : jj);
        kk = kk < 0 ? 0 : (kk > snz - 1 ? snz - 1 : kk);
        c.idx[q] = ((int64_t)ii * sny + jj) * snz + kk;
        c.w[q] = wx[a] * wy[b] * wz[e];
        c.dw[q][0] = sgn[a] * inv_dx * wy[b] * wz[e];
        c.dw[q][1] = sgn[b] * inv_dx * wx[a] * wz[e];
        c.dw[q][2] = sgn[e] * inv_dx * wx[a] * wy[b];
        o[q][0] = (ax == 0 ? (float)ii : (float)ii + 0.5f) * dx - px;
        o[q][1] = (ax == 1 ? (float)jj : (float)jj + 0.5f) * dx - py;
        o[q][2] = (ax == 2 ? (float)kk : (float)kk + 0.5f) * dx - pz;
      }
}

__device__ __forceinline__ void adj_g2p_apic_item(const AdjArgs &a, int64_t q) {
  const float4 r0 = a.rec0[q];
  const float p[3] = {r0.x, r0.y, r0.z};
  const float dx = a.dx, inv_dx = 1.0f / dx;
  const float inv = __fdiv_rn(3.0f, dx * dx);
  const float g[3] = {__fdiv_rn(p[0], dx), __fdiv_rn(p[1], dx), __fdiv_rn(p[2], dx)};
  const float h[3] = {g[0] - 0.5f, g[1] - 0.5f, g[2] - 0.5f};
  const int sz[3][3] = {{a.nx + 1, a.ny, a.nz}, {a.nx, a.ny + 1, a.nz}, {a.nx, a.ny, a.nz + 1}};
  const float dom[3] = {a.dom0, a.dom1, a.dom2};
  const float eps = dx * 1.001f;
  // velocity after G2P (for the advection clamp test)
  float vnew[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Corners cs;
    float o[8][3];
    apic_corners(c == 0 ? g[0] : h[0], c == 1 ? g[1] : h[1], c == 2 ? g[2] : h[2], sz[c][0],
                 sz[c][1], sz[c][2], c, dx, inv_dx, p[0], p[1], p[2], cs, o);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += cs.w[k] * a.u3[c][cs.idx[k]];
    vnew[c] = acc;
  }
  float xb[3], vb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float xo = a.xbar_out[3 * q + d], vo = a.vbar_out[3 * q + d];
    const float xn = p[d] + vnew[d] * a.dt;
    const bool free = xn >= eps && xn <= dom[d] - eps;
    xb[d] = free ? xo : 0.0f;
    vb[d] = vo + (free ? a.dt * xo : 0.0f);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Corners cs;
    float o[8][3];
    apic_corners(c == 0 ? g[0] : h[0], c == 1 ? g[1] : h[1], c == 2 ? g[2] : h[2], sz[c][0],
                 sz[c][1], sz[c][2], c, dx, inv_dx, p[0], p[1], p[2], cs, o);
    const float cb[3] = {a.Cbar_out[9 * q + 3 * c], a.Cbar_out[9 * q + 3 * c + 1],
                         a.Cbar_out[9 * q + 3 * c + 2]};
    float su = 0.f;  // sum_f S u3
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float uv = a.u3[c][cs.idx[k]];
      const float gk = vb[c] + inv * (o[k][0] * cb[0] + o[k][1] * cb[1] + o[k][2] * cb[2]);
      atomicAdd(&a.ubar3[c][cs.idx[k]], cs.w[k] * gk);
#pragma unroll
      for (int d = 0; d < 3; ++d) xb[d] += cs.dw[k][d] * uv * gk;
      su += cs.w[k] * uv;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) xb[d] -= inv * su * cb[d];
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) a.xbar_acc[3 * q + d] = xb[d];
}

__global__ void k_adj_g2p_apic(AdjArgs a) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < a.n) adj_g2p_apic_item(a, q);
}

__device__ __forceinline__ void adj_p2g_apic_item(const AdjArgs &a, int64_t q) {
  const float4 r0 = a.rec0[q], r1 = a.rec1[q], r2 = a.rec2[q], r3 = a.rec3[q];
  const float vel[3] = {r1.x, r2.x, r3.x};
  const float C[3][3] = {{r1.y, r1.z, r1.w}, {r2.y, r2.z, r2.w}, {r3.y, r3.z, r3.w}};
  const float p[3] = {r0.x, r0.y, r0.z};
  const float dx = a.dx, inv_dx = 1.0f / dx;
  const float g[3] = {__fdiv_rn(p[0], dx), __fdiv_rn(p[1], dx), __fdiv_rn(p[2], dx)};
  const float h[3] = {g[0] - 0.5f, g[1] - 0.5f, g[2] - 0.5f};
  const int sz[3][3] = {{a.nx + 1, a.ny, a.nz}, {a.nx, a.ny + 1, a.nz}, {a.nx, a.ny, a.nz + 1}};
  float xb[3] = {a.xbar_acc[3 * q], a.xbar_acc[3 * q + 1], a.xbar_acc[3 * q + 2]};
  float vb[3] = {0.f, 0.f, 0.f};
  float Cb[3][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Corners cs;
    scatter_corners(c == 0 ? g[0] : h[0], c == 1 ? g[1] : h[1], c == 2 ? g[2] : h[2], sz[c][0],
                    sz[c][1], sz[c][2], inv_dx, cs);
    const int i0 = __float2int_rz(floorf(c == 0 ? g[0] : h[0])),
              j0 = __float2int_rz(floorf(c == 1 ? g[1] : h[1])),
              k0 = __float2int_rz(floorf(c == 2 ? g[2] : h[2]));
    float wqs = 0.f;  // sum_f W qbar
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (cs.idx[k] < 0) continue;
      const int ii = i0 + (k >> 2), jj = j0 + ((k >> 1) & 1), kk = k0 + (k & 1);
      const float o[3] = {(c == 0 ? (float)ii : (float)ii + 0.5f) * dx - p[0],
                          (c == 1 ? (float)jj : (float)jj + 0.5f) * dx - p[1],
                          (c == 2 ? (float)kk : (float)kk + 0.5f) * dx - p[2]};
      const float qb = a.qbar[c][cs.idx[k]], mb = a.mbar[c][cs.idx[k]];
      const float val = vel[c] + C[c][0] * o[0] + C[c][1] * o[1] + C[c][2] * o[2];
      const float wq = cs.w[k] * qb;
      vb[c] += wq;
      wqs += wq;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        Cb[c][d] += wq * o[d];
        xb[d] += cs.dw[k][d] * (val * qb + mb);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) xb[d] -= wqs * C[c][d];
  }
  const int64_t s = a.order[q];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    a.xbar_in[3 * s + d] = xb[d];
    a.vbar_in[3 * s + d] = vb[d];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) a.Cbar_in[9 * s + 3 * c + d] = Cb[c][d];
}

__global__ void k_adj_p2g_apic(AdjArgs a) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < a.n) adj_p2g_apic_item(a, q);
}

// ---- batches: each item finds its scene and runs the single-grid body on
// the scene's view of the concatenated arrays (particles stay global).
__device__ __forceinline__ AdjArgs adj_view(const AdjArgs &a, const SegRow &r) {
  AdjArgs v = a;
  const int64_t off[3] = {r.fu0, r.fv0, r.fw0};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v.m[c] = a.m[c] + off[c];
    v.un[c] = a.un[c] + off[c];
    v.u3[c] = a.u3[c] + off[c];
    v.ubar3[c] = a.ubar3[c] + off[c];
    v.qbar[c] = a.qbar[c] + off[c];
    v.mbar[c] = a.mbar[c] + off[c];
  }
  v.label = a.label + r.cell0;
  v.div_io = a.div_io + r.cell0;
  v.lambda = a.lambda + r.cell0;
  v.dx = r.dx;
  v.dom0 = r.dom0; v.dom1 = r.dom1; v.dom2 = r.dom2;
  v.nx = r.nx; v.ny = r.ny; v.nz = r.nz;
  return v;
}

template <int KIND>  // 0 g2p, 1 p2g, 2 g2p apic, 3 p2g apic
__global__ void kb_adj_particles(AdjArgs a, SegIndex sx) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= a.n) return;
  const AdjArgs v = adj_view(a, sx.row[seg_find(sx.part0, sx.n, q)]);
  if (KIND == 0) adj_g2p_item(v, q);
  if (KIND == 1) adj_p2g_item(v, q);
  if (KIND == 2) adj_g2p_apic_item(v, q);
  if (KIND == 3) adj_p2g_apic_item(v, q);
}

__global__ void kb_adj_grad(AdjArgs a, SegIndex sx, int64_t ncell, float rho, float dt) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell;
       c += (int64_t)gridDim.x * blockDim.x) {
    const SegRow r = sx.row[seg_find(sx.cell0, sx.n, c)];
    float k = rho * r.dx;  // dt / (rho dx) per scene
    k = dt / k;
    adj_grad_item(adj_view(a, r), c - r.cell0, k);
  }
}

__global__ void kb_adj_faces(AdjArgs a, SegIndex sx, int64_t nslot, float rho, float dt) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nslot;
       t += (int64_t)gridDim.x * blockDim.x) {
    const SegRow r = sx.row[seg_find(sx.fslot0, sx.n, t)];
    float s = rho * r.dx;  // (rho dx) / dt per scene
    s = s / dt;
    adj_faces_item(adj_view(a, r), t - r.fslot0, s);
  }
}

// ---- density splat (meshing/surface.py:14-43) and control sampling -------
__global__ void k_splat(const float *__restrict__ pos, int64_t n, float dx, int nx, int ny,
                        int nz, float *rho) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], dx) - 0.5f, nx, ny, nz, 1.0f / dx, cs);
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (cs.idx[k] >= 0) atomicAdd(&rho[cs.idx[k]], cs.w[k]);
}

__global__ void k_splat_adj(const float *__restrict__ pos, int64_t n, float dx, int nx, int ny,
                            int nz, const float *__restrict__ rho_bar, float *pos_bar) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], dx) - 0.5f, nx, ny, nz, 1.0f / dx, cs);
  float xb[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (cs.idx[k] < 0) continue;
    const float rb = rho_bar[cs.idx[k]];
#pragma unroll
    for (int d = 0; d < 3; ++d) xb[d] += cs.dw[k][d] * rb;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) pos_bar[3 * q + d] = xb[d];
}

// v_p = sum_c N_pc U_c of a cell-centred 3-component field (3, nx, ny, nz).
__global__ void k_sample_cells(const float *__restrict__ grid3, const float *__restrict__ pos,
                               int64_t n, float dx, int nx, int ny, int nz, float *vel) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], dx) - 0.5f, nx, ny, nz, 1.0f / dx, cs);
  const int64_t ncell = (int64_t)nx * ny * nz;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (cs.idx[k] >= 0) acc += cs.w[k] * grid3[d * ncell + cs.idx[k]];
    vel[3 * q + d] = acc;
  }
}

__global__ void k_sample_cells_adj(const float *__restrict__ pos, int64_t n, float dx, int nx,
                                   int ny, int nz, const float *__restrict__ vel_bar,
                                   float *grid3_bar) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], dx) - 0.5f, nx, ny, nz, 1.0f / dx, cs);
  const int64_t ncell = (int64_t)nx * ny * nz;
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (cs.idx[k] >= 0) atomicAdd(&grid3_bar[d * ncell + cs.idx[k]], cs.w[k] * vel_bar[3 * q + d]);
}

// Over a batch: particle i belongs to the scene of the particle prefix, the
// cell arrays are the scenes' arrays concatenated, and a control field holds
// each scene's (3, nx, ny, nz) block at 3 * cell0.
__global__ void kb_splat(const float *__restrict__ pos, int64_t n, SegIndex sx, float *rho) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SegRow r = sx.row[seg_find(sx.part0, sx.n, q)];
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], r.dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], r.dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], r.dx) - 0.5f, r.nx, r.ny, r.nz, 1.0f / r.dx, cs);
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (cs.idx[k] >= 0) atomicAdd(&rho[r.cell0 + cs.idx[k]], cs.w[k]);
}

__global__ void kb_splat_adj(const float *__restrict__ pos, int64_t n, SegIndex sx,
                             const float *__restrict__ rho_bar, float *pos_bar) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SegRow r = sx.row[seg_find(sx.part0, sx.n, q)];
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], r.dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], r.dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], r.dx) - 0.5f, r.nx, r.ny, r.nz, 1.0f / r.dx, cs);
  float xb[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (cs.idx[k] < 0) continue;
    const float rb = rho_bar[r.cell0 + cs.idx[k]];
#pragma unroll
    for (int d = 0; d < 3; ++d) xb[d] += cs.dw[k][d] * rb;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) pos_bar[3 * q + d] = xb[d];
}

__global__ void kb_sample_cells(const float *__restrict__ grid3, const float *__restrict__ pos,
                                int64_t n, SegIndex sx, float *vel) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SegRow r = sx.row[seg_find(sx.part0, sx.n, q)];
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], r.dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], r.dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], r.dx) - 0.5f, r.nx, r.ny, r.nz, 1.0f / r.dx, cs);
  const int64_t nc = (int64_t)r.nx * r.ny * r.nz;
  const float *g = grid3 + 3 * r.cell0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (cs.idx[k] >= 0) acc += cs.w[k] * g[d * nc + cs.idx[k]];
    vel[3 * q + d] = acc;
  }
}

__global__ void kb_sample_cells_adj(const float *__restrict__ pos, int64_t n, SegIndex sx,
                                    const float *__restrict__ vel_bar, float *grid3_bar) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= n) return;
  const SegRow r = sx.row[seg_find(sx.part0, sx.n, q)];
  Corners cs;
  scatter_corners(__fdiv_rn(pos[3 * q], r.dx) - 0.5f, __fdiv_rn(pos[3 * q + 1], r.dx) - 0.5f,
                  __fdiv_rn(pos[3 * q + 2], r.dx) - 0.5f, r.nx, r.ny, r.nz, 1.0f / r.dx, cs);
  const int64_t nc = (int64_t)r.nx * r.ny * r.nz;
  float *g = grid3_bar + 3 * r.cell0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (cs.idx[k] >= 0) atomicAdd(&g[d * nc + cs.idx[k]], cs.w[k] * vel_bar[3 * q + d]);
}

// ---- record layout -------------------------------------------------------
struct RecordLayout {
  size_t rec0, rec1, rec2, rec3, order, m[3], un[3], u3[3], label, bytes;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static RecordLayout layout(const Ctx *c) {
  RecordLayout L{};
  const int64_t n = c->p.n;
  const int64_t fsz[3] = {c->nu, c->nv, c->nw};  // all scenes' faces of a batch
  size_t o = 0;
  L.rec0 = o; o = align256(o + n * 16);
  L.rec1 = o; o = align256(o + n * 16);
  L.rec2 = o; o = align256(o + n * 16);  // APIC: the rest of the input C
  L.rec3 = o; o = align256(o + n * 16);
  L.order = o; o = align256(o + n * 4);
  for (int q = 0; q < 3; ++q) { L.m[q] = o; o = align256(o + fsz[q] * 4); }
  for (int q = 0; q < 3; ++q) { L.un[q] = o; o = align256(o + fsz[q] * 4); }
  for (int q = 0; q < 3; ++q) { L.u3[q] = o; o = align256(o + fsz[q] * 4); }
  L.label = o; o = align256(o + c->ncell);
  L.bytes = o;
  return L;
}

static int adj_reserve(Ctx *c) {
  const int64_t nf = c->nfslot;  // face slots: >= the faces of each component
  const int64_t need_f = 9 * nf, need_p = 3 * (c->p.n > 0 ? c->p.n : 1);
  if (c->adj_faces && c->adj_faces_n >= need_f && c->adj_part_n >= need_p) return GF_OK;
  if (c->adj_faces) cudaFree(c->adj_faces);
  if (c->adj_part) cudaFree(c->adj_part);
  c->adj_faces = nullptr;
  c->adj_part = nullptr;
  int e = check_cuda(c, cudaMalloc(&c->adj_faces, need_f * 4), "alloc adjoint faces");
  if (e) return e;
  if ((e = check_cuda(c, cudaMalloc(&c->adj_part, need_p * 4), "alloc adjoint particles")))
    return e;
  c->adj_faces_n = need_f;
  c->adj_part_n = need_p;
  return GF_OK;
}

static bool pic_only(const gf_step_params *prm) {
  return prm->transfer != GF_APIC && prm->flip_blend == 0.0f;
}

// Transfers the recorded substep can be differentiated for: PIC (flip_blend
// 0) and APIC.
static bool adjointable(const gf_step_params *prm) {
  return pic_only(prm) || prm->transfer == GF_APIC;
}

}  // namespace gf

using gf::Ctx;

extern "C" {

int gf_record_bytes(void *ctx, int64_t *bytes) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !bytes) return GF_INVALID_ARG;
  if (!c->bound) return gf::fail(c, GF_INVALID_ARG, "gf_record_bytes: buffers not bound");
  *bytes = (int64_t)gf::layout(c).bytes;
  return GF_OK;
}

int gf_step_record(void *ctx, const gf_step_params *prm, void *record) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !prm || !record) return GF_INVALID_ARG;
  if (!gf::adjointable(prm))
    return gf::fail(c, GF_INVALID_ARG, "the adjoint substep supports PIC (flip_blend 0) and APIC");
  int e = gf_step(ctx, prm);
  if (e) return e;
  const gf::RecordLayout L = gf::layout(c);
  char *r = static_cast<char *>(record);
  cudaStream_t st = c->stream;
  const int64_t n = c->p.n;
  const int64_t fsz[3] = {c->nu, c->nv, c->nw};
  const float *mw[3] = {c->f.uw, c->f.vw, c->f.ww}, *us[3] = {c->f.us, c->f.vs, c->f.ws},
              *u3[3] = {c->f.u, c->f.v, c->f.w};
  // 6 particle/label copies + (m, un, u3) per component
  constexpr int kCopies = 6 + 3 * 3;
  const size_t crec = prm->transfer == GF_APIC ? (size_t)n * 16 : 0;
  struct { size_t off; const void *src; size_t bytes; } cp[kCopies] = {
      {L.rec0, c->rec0, (size_t)n * 16}, {L.rec1, c->rec1, (size_t)n * 16},
      {L.rec2, c->rec2, crec}, {L.rec3, c->rec3, crec},
      {L.order, c->order, (size_t)n * 4}, {L.label, c->f.label, (size_t)c->ncell}};
  int k = 6;
  for (int q = 0; q < 3; ++q) {
    cp[k++] = {L.m[q], mw[q], (size_t)fsz[q] * 4};
    cp[k++] = {L.un[q], us[q], (size_t)fsz[q] * 4};
    cp[k++] = {L.u3[q], u3[q], (size_t)fsz[q] * 4};
  }
  for (auto &x : cp)
    if (x.bytes && (e = gf::check_cuda(c, cudaMemcpyAsync(r + x.off, x.src, x.bytes,
                                                          cudaMemcpyDeviceToDevice, st),
                                       "gf_step_record copy")))
      return e;
  return GF_OK;
}

}  // extern "C"

namespace gf {

// One substep's adjoint (PIC or APIC kernels around the shared grid part).
static int step_adjoint(Ctx *c, const gf_step_params *prm, const void *record,
                        const float *xbar_out, const float *vbar_out, const float *Cbar_out,
                        float *xbar_in, float *vbar_in, float *Cbar_in, bool apic) {
  int e = adj_reserve(c);
  if (e) return e;
  const RecordLayout L = layout(c);
  const char *r = static_cast<const char *>(record);
  cudaStream_t st = c->stream;
  const int64_t n = c->p.n;
  const int64_t nfmax = c->nfslot;
  AdjArgs a{};
  a.rec0 = reinterpret_cast<const float4 *>(r + L.rec0);
  a.rec1 = reinterpret_cast<const float4 *>(r + L.rec1);
  a.rec2 = reinterpret_cast<const float4 *>(r + L.rec2);
  a.rec3 = reinterpret_cast<const float4 *>(r + L.rec3);
  a.Cbar_out = Cbar_out;
  a.Cbar_in = Cbar_in;
  a.order = reinterpret_cast<const int32_t *>(r + L.order);
  a.label = reinterpret_cast<const uint8_t *>(r + L.label);
  for (int q = 0; q < 3; ++q) {
    a.m[q] = reinterpret_cast<const float *>(r + L.m[q]);
    a.un[q] = reinterpret_cast<const float *>(r + L.un[q]);
    a.u3[q] = reinterpret_cast<const float *>(r + L.u3[q]);
    a.ubar3[q] = c->adj_faces + q * nfmax;
    a.qbar[q] = c->adj_faces + (3 + q) * nfmax;
    a.mbar[q] = c->adj_faces + (6 + q) * nfmax;
  }
  a.div_io = c->f.div;
  a.lambda = c->f.p;
  a.xbar_out = xbar_out;
  a.vbar_out = vbar_out;
  a.xbar_acc = c->adj_part;
  a.xbar_in = xbar_in;
  a.vbar_in = vbar_in;
  a.n = n;
  a.dx = c->dx;
  a.dt = prm->dt;
  a.rho = prm->rho;
  a.dom0 = c->dom[0];
  a.dom1 = c->dom[1];
  a.dom2 = c->dom[2];
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  if ((e = check_cuda(c, cudaMemsetAsync(c->adj_faces, 0, 3 * nfmax * 4, st), "zero ubar")))
    return e;
  const unsigned gp = (unsigned)((n + 255) / 256);
  const bool batch = c->nseg > 0;
  const SegIndex sx = batch ? seg_index(c) : SegIndex{};
  if (n > 0) {
    if (batch && apic)
      kb_adj_particles<2><<<gp, 256, 0, st>>>(a, sx);
    else if (batch)
      kb_adj_particles<0><<<gp, 256, 0, st>>>(a, sx);
    else if (apic)
      k_adj_g2p_apic<<<gp, 256, 0, st>>>(a);
    else
      k_adj_g2p<<<gp, 256, 0, st>>>(a);
    c->launches++;
  }
  // pressure-gradient adjoint -> rhs of the adjoint solve, on the recorded labels
  if ((e = check_cuda(c, cudaMemcpyAsync(c->f.label, a.label, c->ncell,
                                         cudaMemcpyDeviceToDevice, st),
                      "restore labels")))
    return e;
  float kk = prm->rho * c->dx;  // dt / (rho dx), as k3_subtract_pressure_grad
  kk = prm->dt / kk;
  const unsigned gc = (unsigned)((c->ncell + 255) / 256 < (int64_t)c->num_sms * 16
                                     ? (c->ncell + 255) / 256
                                     : (int64_t)c->num_sms * 16);
  if (batch)
    kb_adj_grad<<<gc, 256, 0, st>>>(a, sx, c->ncell, prm->rho, prm->dt);
  else
    k_adj_grad<<<gc, 256, 0, st>>>(a, kk);
  c->launches++;
  // A lambda = pbar with the same SPD operator (labels fixed)
  gf_step_params sp = *prm;
  sp.rhs_sign = 1;
  if (sp.solver != GF_PCG && sp.solver != GF_PCG_REFINED) sp.solver = GF_PCG;
  if ((e = launch_pressure(c, &sp))) return e;
  float s = prm->rho * c->dx;  // (rho dx) / dt, as k3_compute_divergence
  s = s / prm->dt;
  const unsigned gf_ = (unsigned)((nfmax + 255) / 256 < (int64_t)c->num_sms * 16
                                      ? (nfmax + 255) / 256
                                      : (int64_t)c->num_sms * 16);
  if (batch)
    kb_adj_faces<<<gf_, 256, 0, st>>>(a, sx, c->nfslot, prm->rho, prm->dt);
  else
    k_adj_faces<<<gf_, 256, 0, st>>>(a, s);
  c->launches++;
  if (n > 0) {
    if (batch && apic)
      kb_adj_particles<3><<<gp, 256, 0, st>>>(a, sx);
    else if (batch)
      kb_adj_particles<1><<<gp, 256, 0, st>>>(a, sx);
    else if (apic)
      k_adj_p2g_apic<<<gp, 256, 0, st>>>(a);
    else
      k_adj_p2g<<<gp, 256, 0, st>>>(a);
    c->launches++;
  }
  return check_launch(c, apic ? "gf_step_adjoint_apic" : "gf_step_adjoint");
}

}  // namespace gf

extern "C" {

int gf_step_adjoint(void *ctx, const gf_step_params *prm, const void *record,
                    const float *xbar_out, const float *vbar_out, float *xbar_in, float *vbar_in) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !prm || !record || !xbar_out || !vbar_out || !xbar_in || !vbar_in)
    return GF_INVALID_ARG;
  if (!c->bound) return gf::fail(c, GF_INVALID_ARG, "gf_step_adjoint: buffers not bound");
  if (!gf::pic_only(prm))
    return gf::fail(c, GF_INVALID_ARG,
                    "gf_step_adjoint is the PIC (flip_blend 0) adjoint; APIC uses "
                    "gf_step_adjoint_apic");
  return gf::step_adjoint(c, prm, record, xbar_out, vbar_out, nullptr, xbar_in, vbar_in, nullptr,
                          false);
}

int gf_step_adjoint_apic(void *ctx, const gf_step_params *prm, const void *record,
                         const float *xbar_out, const float *vbar_out, const float *Cbar_out,
                         float *xbar_in, float *vbar_in, float *Cbar_in) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !prm || !record || !xbar_out || !vbar_out || !Cbar_out || !xbar_in || !vbar_in ||
      !Cbar_in)
    return GF_INVALID_ARG;
  if (!c->bound) return gf::fail(c, GF_INVALID_ARG, "gf_step_adjoint_apic: buffers not bound");
  if (prm->transfer != GF_APIC)
    return gf::fail(c, GF_INVALID_ARG, "gf_step_adjoint_apic needs an APIC substep");
  return gf::step_adjoint(c, prm, record, xbar_out, vbar_out, Cbar_out, xbar_in, vbar_in, Cbar_in,
                          true);
}

int gf_density_splat(void *ctx, const float *pos, int64_t n, float *rho) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || (n > 0 && !pos) || !rho) return GF_INVALID_ARG;
  int e = gf::check_cuda(c, cudaMemsetAsync(rho, 0, c->ncell * 4, c->stream), "zero rho");
  if (e || n == 0) return e;
  if (c->nseg) {
    if (n != c->p.n) return gf::fail(c, GF_INVALID_ARG, "batch splat: n must be the bound count");
    gf::kb_splat<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(pos, n, gf::seg_index(c),
                                                                     rho);
  } else {
    gf::k_splat<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(pos, n, c->dx, c->nx, c->ny,
                                                                    c->nz, rho);
  }
  c->launches++;
  return gf::check_launch(c, "gf_density_splat");
}

int gf_density_splat_adjoint(void *ctx, const float *pos, int64_t n, const float *rho_bar,
                             float *pos_bar) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || (n > 0 && (!pos || !pos_bar)) || !rho_bar) return GF_INVALID_ARG;
  if (n == 0) return GF_OK;
  if (c->nseg) {
    if (n != c->p.n) return gf::fail(c, GF_INVALID_ARG, "batch splat: n must be the bound count");
    gf::kb_splat_adj<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        pos, n, gf::seg_index(c), rho_bar, pos_bar);
  } else {
    gf::k_splat_adj<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        pos, n, c->dx, c->nx, c->ny, c->nz, rho_bar, pos_bar);
  }
  c->launches++;
  return gf::check_launch(c, "gf_density_splat_adjoint");
}

int gf_sample_cells(void *ctx, const float *grid3, const float *pos, int64_t n, float *vel) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !grid3 || (n > 0 && (!pos || !vel))) return GF_INVALID_ARG;
  if (n == 0) return GF_OK;
  if (c->nseg) {
    if (n != c->p.n) return gf::fail(c, GF_INVALID_ARG, "batch sampling: n must be the bound count");
    gf::kb_sample_cells<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        grid3, pos, n, gf::seg_index(c), vel);
  } else {
    gf::k_sample_cells<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        grid3, pos, n, c->dx, c->nx, c->ny, c->nz, vel);
  }
  c->launches++;
  return gf::check_launch(c, "gf_sample_cells");
}

int gf_sample_cells_adjoint(void *ctx, const float *pos, int64_t n, const float *vel_bar,
                            float *grid3_bar) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !grid3_bar || (n > 0 && (!pos || !vel_bar))) return GF_INVALID_ARG;
  int e = gf::check_cuda(c, cudaMemsetAsync(grid3_bar, 0, 3 * c->ncell * 4, c->stream),
                         "zero grid bar");
  if (e || n == 0) return e;
  if (c->nseg) {
    if (n != c->p.n) return gf::fail(c, GF_INVALID_ARG, "batch sampling: n must be the bound count");
    gf::kb_sample_cells_adj<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        pos, n, gf::seg_index(c), vel_bar, grid3_bar);
  } else {
    gf::k_sample_cells_adj<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
        pos, n, c->dx, c->nx, c->ny, c->nz, vel_bar, grid3_bar);
  }
  c->launches++;
  return gf::check_launch(c, "gf_sample_cells_adjoint");
}

}  // extern "C"
