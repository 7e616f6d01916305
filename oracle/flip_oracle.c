/*
 * CPU oracle for the FLIP/PIC/APIC substep (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, never the product: only tests/, the smoke check
 * and bench.py's CPU-baseline / reference arm load it.  It restates, in plain
 * C and in the same float32 operation order, the reference kernels of
 * src/gpufluid/solvers/solver3d.py and src/gpufluid/primitives/gridmath.py so
 * that, run sequentially (par == 0), its output is bit-identical to the
 * reference's own source executed with threads in launch order (see
 * tests/golden/make_golden.py).  Compile with -ffp-contract=off and without
 * -ffast-math: every a*b+c must round twice, as in the reference.
 *
 * par != 0 selects OpenMP loops (grid kernels in parallel, P2G with atomic
 * adds, dot products as reductions): the CPU baseline timing mode.  Results
 * then differ from the sequential mode only by floating-point summation order.
 *
 * Layout (same as the reference, C order [i][j][k], k fastest):
 *   u (nx+1, ny, nz)   v (nx, ny+1, nz)   w (nx, ny, nz+1)
 *   cell arrays (nx, ny, nz); marker int32: 0 air, 1 fluid, 2 solid
 *   particles: pos, vel (P, 3) float32; C (P, 3, 3) float32 row-major
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UIDX(i, j, k) (((int64_t)(i) * ny + (j)) * nz + (k))
#define VIDX(i, j, k) (((int64_t)(i) * (ny + 1) + (j)) * nz + (k))
#define WIDX(i, j, k) (((int64_t)(i) * ny + (j)) * (nz + 1) + (k))
#define CIDX(i, j, k) (((int64_t)(i) * ny + (j)) * nz + (k))

static int clamp_int(int v, int lo, int hi) { /* gridmath.py:12-17 */
  if (v < lo) return lo;
  if (v > hi) return hi;
  return v;
}
static float clampf(float x, float lo, float hi) {
  if (x < lo) return lo;
  if (x > hi) return hi;
  return x;
}

int og_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* k3_clear_grid, solver3d.py:41-65 */
void og_clear_grid(int nx, int ny, int nz, float *u, float *v, float *w, float *uw,
                   float *vw, float *ww, int32_t *marker) {
  int64_t nu = (int64_t)(nx + 1) * ny * nz, nv = (int64_t)nx * (ny + 1) * nz,
          nw = (int64_t)nx * ny * (nz + 1), nc = (int64_t)nx * ny * nz;
  memset(u, 0, nu * 4); memset(uw, 0, nu * 4);
  memset(v, 0, nv * 4); memset(vw, 0, nv * 4);
  memset(w, 0, nw * 4); memset(ww, 0, nw * 4);
  for (int64_t c = 0; c < nc; ++c)
    if (marker[c] != 2) marker[c] = 0;
}

/* scatter_face, gridmath.py:70-95 (8-corner trilinear scatter). */
static void scatter_face(float *field, float *weight, float val, float fx, float fy,
                         float fz, int snx, int sny, int snz, int par) {
  float fi = floorf(fx), fj = floorf(fy), fk = floorf(fz);
  int i0 = (int)fi, j0 = (int)fj, k0 = (int)fk;
  float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        int ii = i0 + di, jj = j0 + dj, kk = k0 + dk;
        if (ii >= 0 && ii < snx && jj >= 0 && jj < sny && kk >= 0 && kk < snz) {
          float wxi = di == 0 ? 1.0f - sx : sx;
          float wyi = dj == 0 ? 1.0f - sy : sy;
          float wzi = dk == 0 ? 1.0f - sz : sz;
          float wgt = wxi * wyi;
          wgt = wgt * wzi;
          int64_t idx = ((int64_t)ii * sny + jj) * snz + kk;
          float add = val * wgt;
          if (par) {
#pragma omp atomic
            field[idx] += add;
#pragma omp atomic
            weight[idx] += wgt;
          } else {
            field[idx] = field[idx] + add;
            weight[idx] = weight[idx] + wgt;
          }
        }
      }
}

static int cell_of(float p, float dx, int n) { /* int(p / dx) clamped */
  float q = p / dx;
  return clamp_int((int)q, 0, n - 1);
}

/* k3_p2g, solver3d.py:72-114 */
void og_p2g_flip(int nx, int ny, int nz, float dx, int64_t P, const float *pos,
                 const float *vel, float *u, float *v, float *w, float *uw, float *vw,
                 float *ww, int32_t *marker, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int64_t pid = 0; pid < P; ++pid) {
    float px = pos[3 * pid], py = pos[3 * pid + 1], pz = pos[3 * pid + 2];
    int ci = cell_of(px, dx, nx), cj = cell_of(py, dx, ny), ck = cell_of(pz, dx, nz);
    if (marker[CIDX(ci, cj, ck)] != 2) marker[CIDX(ci, cj, ck)] = 1;
    float fx = px / dx - 0.0f, fy = py / dx - 0.0f, fz = pz / dx - 0.0f;
    scatter_face(u, uw, vel[3 * pid + 0], fx, fy - 0.5f, fz - 0.5f, nx + 1, ny, nz, par);
    scatter_face(v, vw, vel[3 * pid + 1], fx - 0.5f, fy, fz - 0.5f, nx, ny + 1, nz, par);
    scatter_face(w, ww, vel[3 * pid + 2], fx - 0.5f, fy - 0.5f, fz, nx, ny, nz + 1, par);
  }
}

/* One APIC face component of k3_p2g_apic, solver3d.py:1510-1588.  (ox0, oy0,
 * oz0) = 1 if that axis is the face-normal axis (world offset ii*dx), else 0
 * (world offset (ii+0.5)*dx). */
static void apic_scatter(float *field, float *weight, float vp, const float *Crow,
                         float px, float py, float pz, float dx, float fx, float fy,
                         float fz, int snx, int sny, int snz, int ax, int par) {
  int i0 = (int)floorf(fx), j0 = (int)floorf(fy), k0 = (int)floorf(fz);
  float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
      for (int dk = 0; dk < 2; ++dk) {
        int ii = i0 + di, jj = j0 + dj, kk = k0 + dk;
        if (ii >= 0 && ii < snx && jj >= 0 && jj < sny && kk >= 0 && kk < snz) {
          float wxi = di == 0 ? 1.0f - sx : sx;
          float wyi = dj == 0 ? 1.0f - sy : sy;
          float wzi = dk == 0 ? 1.0f - sz : sz;
          float wt = wxi * wyi;
          wt = wt * wzi;
          float ox = ax == 0 ? (float)ii * dx - px : ((float)ii + 0.5f) * dx - px;
          float oy = ax == 1 ? (float)jj * dx - py : ((float)jj + 0.5f) * dx - py;
          float oz = ax == 2 ? (float)kk * dx - pz : ((float)kk + 0.5f) * dx - pz;
          float t0 = Crow[0] * ox, t1 = Crow[1] * oy, t2 = Crow[2] * oz;
          float ueff = vp + t0;
          ueff = ueff + t1;
          ueff = ueff + t2;
          int64_t idx = ((int64_t)ii * sny + jj) * snz + kk;
          float add = ueff * wt;
          if (par) {
#pragma omp atomic
            field[idx] += add;
#pragma omp atomic
            weight[idx] += wt;
          } else {
            field[idx] = field[idx] + add;
            weight[idx] = weight[idx] + wt;
          }
        }
      }
}

/* k3_p2g_apic, solver3d.py:1475-1588 */
void og_p2g_apic(int nx, int ny, int nz, float dx, int64_t P, const float *pos,
                 const float *vel, const float *C, float *u, float *v, float *w,
                 float *uw, float *vw, float *ww, int32_t *marker, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int64_t pid = 0; pid < P; ++pid) {
    float px = pos[3 * pid], py = pos[3 * pid + 1], pz = pos[3 * pid + 2];
    const float *Cp = C + 9 * pid;
    int ci = cell_of(px, dx, nx), cj = cell_of(py, dx, ny), ck = cell_of(pz, dx, nz);
    if (marker[CIDX(ci, cj, ck)] != 2) marker[CIDX(ci, cj, ck)] = 1;
    float gx = px / dx, gy = py / dx, gz = pz / dx;
    float hx = gx - 0.5f, hy = gy - 0.5f, hz = gz - 0.5f;
    apic_scatter(u, uw, vel[3 * pid + 0], Cp + 0, px, py, pz, dx, gx - 0.0f, hy - 0.0f,
                 hz - 0.0f, nx + 1, ny, nz, 0, par);
    apic_scatter(v, vw, vel[3 * pid + 1], Cp + 3, px, py, pz, dx, hx - 0.0f, gy - 0.0f,
                 hz - 0.0f, nx, ny + 1, nz, 1, par);
    apic_scatter(w, ww, vel[3 * pid + 2], Cp + 6, px, py, pz, dx, hx - 0.0f, hy - 0.0f,
                 gz - 0.0f, nx, ny, nz + 1, 2, par);
  }
}

/* k3_normalize, solver3d.py:121-142 */
static void normalize_one(float *f, const float *wgt, float *saved, int64_t n, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int64_t i = 0; i < n; ++i) {
    f[i] = wgt[i] > 1.0e-8f ? f[i] / wgt[i] : 0.0f;
    saved[i] = f[i];
  }
}
void og_normalize(int nx, int ny, int nz, float *u, float *v, float *w, const float *uw,
                  const float *vw, const float *ww, float *us, float *vs, float *ws,
                  int par) {
  normalize_one(u, uw, us, (int64_t)(nx + 1) * ny * nz, par);
  normalize_one(v, vw, vs, (int64_t)nx * (ny + 1) * nz, par);
  normalize_one(w, ww, ws, (int64_t)nx * ny * (nz + 1), par);
}

/* k3_add_gravity, solver3d.py:149-156 */
void og_add_gravity(int nx, int ny, int nz, float *v, float g, float dt, int par) {
  int64_t n = (int64_t)nx * (ny + 1) * nz;
#pragma omp parallel for schedule(static) if (par)
  for (int64_t i = 0; i < n; ++i) {
    float gd = g * dt;
    v[i] = v[i] + gd;
  }
}

/* k3_enforce_solid_bc, solver3d.py:758-799 (static solids: zero velocity when
 * solid_* is NULL). */
void og_enforce_bc(int nx, int ny, int nz, float *u, float *v, float *w,
                   const int32_t *marker, const float *solid_u, const float *solid_v,
                   const float *solid_w, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny; ++j)
      for (int k = 0; k <= nz; ++k) {
        if (i <= nx && j < ny && k < nz) {
          int left = (i == 0) || (i > 0 && marker[CIDX(i - 1, j, k)] == 2);
          int right = (i == nx) || (i < nx && marker[CIDX(i, j, k)] == 2);
          if (left || right) u[UIDX(i, j, k)] = solid_u ? solid_u[UIDX(i, j, k)] : 0.0f;
        }
        if (i < nx && j <= ny && k < nz) {
          int bot = (j == 0) || (j > 0 && marker[CIDX(i, j - 1, k)] == 2);
          int top = (j == ny) || (j < ny && marker[CIDX(i, j, k)] == 2);
          if (bot || top) v[VIDX(i, j, k)] = solid_v ? solid_v[VIDX(i, j, k)] : 0.0f;
        }
        if (i < nx && j < ny && k <= nz) {
          int back = (k == 0) || (k > 0 && marker[CIDX(i, j, k - 1)] == 2);
          int front = (k == nz) || (k < nz && marker[CIDX(i, j, k)] == 2);
          if (back || front) w[WIDX(i, j, k)] = solid_w ? solid_w[WIDX(i, j, k)] : 0.0f;
        }
      }
}

/* k3_compute_divergence, solver3d.py:846-871 */
void og_divergence(int nx, int ny, int nz, const float *u, const float *v,
                   const float *w, float *div, const int32_t *marker, float dx, float dt,
                   float rho, int par) {
  float scale = rho * dx;
  scale = scale / dt;
#pragma omp parallel for schedule(static) if (par)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        int64_t c = CIDX(i, j, k);
        if (marker[c] != 1) { div[c] = 0.0f; continue; }
        float d = u[UIDX(i + 1, j, k)] - u[UIDX(i, j, k)];
        d = d + v[VIDX(i, j + 1, k)];
        d = d - v[VIDX(i, j, k)];
        d = d + w[WIDX(i, j, k + 1)];
        d = d - w[WIDX(i, j, k)];
        div[c] = d * scale;
      }
}

/* Neighbour sum / diagonal of the 7-point operator shared by k3_jacobi_pressure
 * (solver3d.py:878-938), k3_gauss_seidel_rb (:1204-1267) and k3_apply_A
 * (:1743-1800). */
static inline void stencil(int nx, int ny, int nz, const int32_t *marker, const float *x,
                           int i, int j, int k, float *sum_out, float *diag_out) {
  float sum = 0.0f, diag = 0.0f;
  int m;
  if (i > 0) { m = marker[CIDX(i - 1, j, k)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i - 1, j, k)]; } }
  if (i < nx - 1) { m = marker[CIDX(i + 1, j, k)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i + 1, j, k)]; } }
  if (j > 0) { m = marker[CIDX(i, j - 1, k)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i, j - 1, k)]; } }
  if (j < ny - 1) { m = marker[CIDX(i, j + 1, k)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i, j + 1, k)]; } }
  if (k > 0) { m = marker[CIDX(i, j, k - 1)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i, j, k - 1)]; } }
  if (k < nz - 1) { m = marker[CIDX(i, j, k + 1)]; if (m != 2) { diag += 1.0f; if (m == 1) sum = sum + x[CIDX(i, j, k + 1)]; } }
  *sum_out = sum;
  *diag_out = diag;
}

/* Jacobi, solver3d.py:878-938 driven as in _step_impl :3594-3599 (p and p_tmp
 * zeroed, iters ping-pong sweeps).  The result is left in p. */
void og_jacobi(int nx, int ny, int nz, float *p, float *p_tmp, const float *div,
               const int32_t *marker, int iters, int par) {
  int64_t nc = (int64_t)nx * ny * nz;
  memset(p, 0, nc * 4);
  memset(p_tmp, 0, nc * 4);
  float *a = p, *b = p_tmp;
  for (int it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(static) if (par)
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          int64_t c = CIDX(i, j, k);
          if (marker[c] != 1) { b[c] = 0.0f; continue; }
          float s, d;
          stencil(nx, ny, nz, marker, a, i, j, k, &s, &d);
          b[c] = d < 0.5f ? 0.0f : (s - div[c]) / d;
        }
    float *t = a; a = b; b = t;
  }
  if (a != p) memcpy(p, a, nc * 4);
}

/* Red-black Gauss-Seidel, solver3d.py:1204-1267, loop :3624-3631. */
void og_gsrb(int nx, int ny, int nz, float *p, const float *div, const int32_t *marker,
             int iters, int par) {
  memset(p, 0, (int64_t)nx * ny * nz * 4);
  for (int it = 0; it < iters; ++it)
    for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static) if (par)
      for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
          for (int k = 0; k < nz; ++k) {
            if ((i + j + k) % 2 != color) continue;
            int64_t c = CIDX(i, j, k);
            if (marker[c] != 1) { p[c] = 0.0f; continue; }
            float s, d;
            stencil(nx, ny, nz, marker, p, i, j, k, &s, &d);
            p[c] = d < 0.5f ? 0.0f : (s - div[c]) / d;
          }
    }
}

static float dot_fluid(int64_t nc, const float *a, const float *b, const int32_t *marker,
                       int par) {
  if (!par) { /* k3_dot_fluid :1859-1871, atomics in thread order */
    float s = 0.0f;
    for (int64_t c = 0; c < nc; ++c)
      if (marker[c] == 1) s = s + a[c] * b[c];
    return s;
  }
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t c = 0; c < nc; ++c)
    if (marker[c] == 1) s += (double)(a[c] * b[c]);
  return (float)s;
}

/* Jacobi-preconditioned CG as driven by _pressure_pcg, solver3d.py:2917-3043
 * (host-synchronised path): cold start, unpreconditioned stop test
 * ||r||^2 < tol^2 ||r0||^2 evaluated every check_every iterations and at the
 * last one.  rhs_sign = +1 reproduces the reference (r0 = +div, which solves
 * A p = +div, the opposite sign of its Jacobi/GS-RB); rhs_sign = -1 solves
 * A p = -div, consistent with Jacobi.  work holds 5 cell arrays.
 * Returns the iteration count the reference reports. */
int og_pcg(int nx, int ny, int nz, float *p, const float *div, const int32_t *marker,
           int max_iter, double tol, int check_every, int rhs_sign, float *work,
           int par, float *rr_out) {
  int64_t nc = (int64_t)nx * ny * nz;
  float *r = work, *z = work + nc, *d = work + 2 * nc, *Ad = work + 3 * nc,
        *diag = work + 4 * nc;
#pragma omp parallel for schedule(static) if (par)
  for (int i = 0; i < nx; ++i) /* k3_compute_diag :1803-1823 */
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        int64_t c = CIDX(i, j, k);
        if (marker[c] != 1) { diag[c] = 1.0f; continue; }
        float s, dg;
        stencil(nx, ny, nz, marker, div, i, j, k, &s, &dg);
        diag[c] = dg > 1.0f ? dg : 1.0f;
      }
  memset(p, 0, nc * 4);
  for (int64_t c = 0; c < nc; ++c) r[c] = rhs_sign > 0 ? div[c] : -div[c];
  for (int64_t c = 0; c < nc; ++c) z[c] = marker[c] != 1 ? 0.0f : r[c] / diag[c];
  memcpy(d, z, nc * 4);
  float rz_old = dot_fluid(nc, r, z, marker, par);
  float r0 = dot_fluid(nc, r, r, marker, par);
  if (rr_out) *rr_out = r0;
  if ((double)r0 < 1e-30) return 0;
  double tol_sq = (tol * tol) * (double)r0;
  for (int it = 0; it < max_iter; ++it) {
#pragma omp parallel for schedule(static) if (par)
    for (int i = 0; i < nx; ++i) /* k3_apply_A */
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          int64_t c = CIDX(i, j, k);
          if (marker[c] != 1) { Ad[c] = 0.0f; continue; }
          float s, dg;
          stencil(nx, ny, nz, marker, d, i, j, k, &s, &dg);
          float t = dg * d[c];
          Ad[c] = t - s;
        }
    float pAp = dot_fluid(nc, d, Ad, marker, par);
    float alpha = fabsf(pAp) < 1.0e-30f ? 0.0f : rz_old / pAp; /* k3_div_scalar */
    float nalpha = alpha * -1.0f;
#pragma omp parallel for schedule(static) if (par)
    for (int64_t c = 0; c < nc; ++c) { /* k3_axpy_devscalar x2 */
      if (marker[c] != 1) { p[c] = 0.0f; r[c] = 0.0f; continue; }
      float t = alpha * d[c];
      p[c] = p[c] + t;
      float q = nalpha * Ad[c];
      r[c] = r[c] + q;
    }
    if ((it + 1) % check_every == 0 || it == max_iter - 1) {
      float rr = dot_fluid(nc, r, r, marker, par);
      if (rr_out) *rr_out = rr;
      if ((double)rr < tol_sq) return it + 1;
    }
#pragma omp parallel for schedule(static) if (par)
    for (int64_t c = 0; c < nc; ++c) z[c] = marker[c] != 1 ? 0.0f : r[c] / diag[c];
    float rz_new = dot_fluid(nc, r, z, marker, par);
    float beta = fabsf(rz_old) < 1.0e-30f ? 0.0f : rz_new / rz_old;
#pragma omp parallel for schedule(static) if (par)
    for (int64_t c = 0; c < nc; ++c) {
      if (marker[c] != 1) { d[c] = 0.0f; continue; }
      float t = beta * d[c];
      d[c] = z[c] + t;
    }
    rz_old = rz_new;
  }
  return max_iter;
}

/* FP64 reference pressure solve: Jacobi-preconditioned CG in double on the
 * same operator (diag = #non-solid neighbours, -1 per fluid neighbour, fluid
 * cells only), solving A p = rhs_sign * div to ||r|| <= tol ||b||.
 * work holds 5 double cell arrays.  Returns iterations, or -1 if max_iter
 * was reached. */
int og_pcg64(int nx, int ny, int nz, double *p, const float *div, const int32_t *marker,
             int max_iter, double tol, int rhs_sign, double *work, double *relres_out) {
  int64_t nc = (int64_t)nx * ny * nz;
  double *r = work, *z = work + nc, *d = work + 2 * nc, *Ad = work + 3 * nc,
         *inv = work + 4 * nc;
  double bb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : bb)
  for (int i = 0; i < nx; ++i)
    for (int j = 0; j < ny; ++j)
      for (int k = 0; k < nz; ++k) {
        int64_t c = CIDX(i, j, k);
        p[c] = 0.0;
        if (marker[c] != 1) { inv[c] = 0.0; r[c] = 0.0; continue; }
        float s, dg;
        stencil(nx, ny, nz, marker, div, i, j, k, &s, &dg);
        inv[c] = 1.0 / (dg > 1.0f ? (double)dg : 1.0);
        r[c] = rhs_sign > 0 ? (double)div[c] : -(double)div[c];
        bb += r[c] * r[c];
      }
  double rz = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz)
  for (int64_t c = 0; c < nc; ++c) { z[c] = r[c] * inv[c]; d[c] = z[c]; rz += r[c] * z[c]; }
  if (bb == 0.0) { if (relres_out) *relres_out = 0.0; return 0; }
  double rr = bb;
  for (int it = 0; it < max_iter; ++it) {
    double pAp = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pAp)
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) {
          int64_t c = CIDX(i, j, k);
          if (marker[c] != 1) { Ad[c] = 0.0; continue; }
          double s = 0.0, dg = 0.0;
          int m;
#define NB(ii, jj, kk, cond) if (cond) { m = marker[CIDX(ii, jj, kk)]; if (m != 2) { dg += 1.0; if (m == 1) s += d[CIDX(ii, jj, kk)]; } }
          NB(i - 1, j, k, i > 0) NB(i + 1, j, k, i < nx - 1) NB(i, j - 1, k, j > 0)
          NB(i, j + 1, k, j < ny - 1) NB(i, j, k - 1, k > 0) NB(i, j, k + 1, k < nz - 1)
#undef NB
          Ad[c] = dg * d[c] - s;
          pAp += d[c] * Ad[c];
        }
    double alpha = rz / pAp, rz_new = 0.0;
    rr = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : rz_new, rr)
    for (int64_t c = 0; c < nc; ++c) {
      p[c] += alpha * d[c];
      r[c] -= alpha * Ad[c];
      z[c] = r[c] * inv[c];
      rz_new += r[c] * z[c];
      rr += r[c] * r[c];
    }
    if (sqrt(rr) <= tol * sqrt(bb)) {
      if (relres_out) *relres_out = sqrt(rr / bb);
      return it + 1;
    }
    double beta = rz_new / rz;
    rz = rz_new;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) d[c] = z[c] + beta * d[c];
  }
  if (relres_out) *relres_out = sqrt(rr / bb);
  return -1;
}

/* k3_subtract_pressure_grad, solver3d.py:1364-1407 */
void og_subtract_grad(int nx, int ny, int nz, float *u, float *v, float *w,
                      const float *p, const int32_t *marker, float dx, float dt,
                      float rho, int par) {
  float scale = rho * dx;
  scale = dt / scale;
#pragma omp parallel for schedule(static) if (par)
  for (int i = 0; i <= nx; ++i)
    for (int j = 0; j <= ny; ++j)
      for (int k = 0; k <= nz; ++k) {
        if (i >= 1 && i <= nx - 1 && j < ny && k < nz) {
          int ml = marker[CIDX(i - 1, j, k)], mr = marker[CIDX(i, j, k)];
          if ((ml == 1 || mr == 1) && ml != 2 && mr != 2) {
            float pl = ml == 1 ? p[CIDX(i - 1, j, k)] : 0.0f;
            float pr = mr == 1 ? p[CIDX(i, j, k)] : 0.0f;
            float g = pr - pl;
            g = scale * g;
            u[UIDX(i, j, k)] = u[UIDX(i, j, k)] - g;
          }
        }
        if (j >= 1 && j <= ny - 1 && i < nx && k < nz) {
          int mb = marker[CIDX(i, j - 1, k)], mt = marker[CIDX(i, j, k)];
          if ((mb == 1 || mt == 1) && mb != 2 && mt != 2) {
            float pb = mb == 1 ? p[CIDX(i, j - 1, k)] : 0.0f;
            float pt = mt == 1 ? p[CIDX(i, j, k)] : 0.0f;
            float g = pt - pb;
            g = scale * g;
            v[VIDX(i, j, k)] = v[VIDX(i, j, k)] - g;
          }
        }
        if (k >= 1 && k <= nz - 1 && i < nx && j < ny) {
          int mba = marker[CIDX(i, j, k - 1)], mfr = marker[CIDX(i, j, k)];
          if ((mba == 1 || mfr == 1) && mba != 2 && mfr != 2) {
            float pba = mba == 1 ? p[CIDX(i, j, k - 1)] : 0.0f;
            float pfr = mfr == 1 ? p[CIDX(i, j, k)] : 0.0f;
            float g = pfr - pba;
            g = scale * g;
            w[WIDX(i, j, k)] = w[WIDX(i, j, k)] - g;
          }
        }
      }
}

/* sample3, gridmath.py:29-63 (clamped trilinear gather). */
static float sample3(const float *f, float fx, float fy, float fz, int nxm, int nym,
                     int nzm) {
  fx = clampf(fx, 0.0f, (float)nxm);
  fy = clampf(fy, 0.0f, (float)nym);
  fz = clampf(fz, 0.0f, (float)nzm);
  int i0 = (int)floorf(fx), j0 = (int)floorf(fy), k0 = (int)floorf(fz);
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
  float sx = clampf(fx - (float)i0, 0.0f, 1.0f);
  float sy = clampf(fy - (float)j0, 0.0f, 1.0f);
  float sz = clampf(fz - (float)k0, 0.0f, 1.0f);
#define F(a, b, c) f[((int64_t)(a) * nym + (b)) * nzm + (c)]
  float c000 = F(i0, j0, k0), c100 = F(i1, j0, k0), c010 = F(i0, j1, k0), c110 = F(i1, j1, k0);
  float c001 = F(i0, j0, k1), c101 = F(i1, j0, k1), c011 = F(i0, j1, k1), c111 = F(i1, j1, k1);
#undef F
  float ox = 1.0f - sx, oy = 1.0f - sy, oz = 1.0f - sz, a, b;
  a = c000 * ox; b = c100 * sx; float c00 = a + b;
  a = c010 * ox; b = c110 * sx; float c10 = a + b;
  a = c001 * ox; b = c101 * sx; float c01 = a + b;
  a = c011 * ox; b = c111 * sx; float c11 = a + b;
  a = c00 * oy; b = c10 * sy; float c0 = a + b;
  a = c01 * oy; b = c11 * sy; float c1 = a + b;
  a = c0 * oz; b = c1 * sz;
  return a + b;
}

static void advect(float *pos, int64_t pid, float nu, float nv, float nw, float dt,
                   float dx, const float *dom) {
  float eps = dx * 1.001f;
  float t;
  t = nu * dt; float x = pos[3 * pid] + t;
  t = nv * dt; float y = pos[3 * pid + 1] + t;
  t = nw * dt; float z = pos[3 * pid + 2] + t;
  pos[3 * pid] = clampf(x, eps, dom[0] - eps);
  pos[3 * pid + 1] = clampf(y, eps, dom[1] - eps);
  pos[3 * pid + 2] = clampf(z, eps, dom[2] - eps);
}

/* k3_g2p_and_advect, solver3d.py:1414-1463 */
void og_g2p_flip(int nx, int ny, int nz, float dx, float dt, float flip_blend,
                 const float *dom, int64_t P, float *pos, float *vel, const float *u,
                 const float *v, const float *w, const float *us, const float *vs,
                 const float *ws, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int64_t pid = 0; pid < P; ++pid) {
    float lx = pos[3 * pid] / dx - 0.0f, ly = pos[3 * pid + 1] / dx - 0.0f,
          lz = pos[3 * pid + 2] / dx - 0.0f;
    float hx = lx - 0.5f, hy = ly - 0.5f, hz = lz - 0.5f;
    float pic_u = sample3(u, lx, hy, hz, nx + 1, ny, nz);
    float old_u = sample3(us, lx, hy, hz, nx + 1, ny, nz);
    float pic_v = sample3(v, hx, ly, hz, nx, ny + 1, nz);
    float old_v = sample3(vs, hx, ly, hz, nx, ny + 1, nz);
    float pic_w = sample3(w, hx, hy, lz, nx, ny, nz + 1);
    float old_w = sample3(ws, hx, hy, lz, nx, ny, nz + 1);
    float du = pic_u - old_u, dv = pic_v - old_v, dw = pic_w - old_w;
    float fu = vel[3 * pid] + du, fv = vel[3 * pid + 1] + dv, fw = vel[3 * pid + 2] + dw;
    float ob = 1.0f - flip_blend, a, b;
    a = flip_blend * fu; b = ob * pic_u; float nu = a + b;
    a = flip_blend * fv; b = ob * pic_v; float nv = a + b;
    a = flip_blend * fw; b = ob * pic_w; float nw = a + b;
    vel[3 * pid] = nu; vel[3 * pid + 1] = nv; vel[3 * pid + 2] = nw;
    advect(pos, pid, nu, nv, nw, dt, dx, dom);
  }
}

/* One face component of k3_g2p_apic_advect, solver3d.py:1626-1724. */
static void apic_gather(const float *f, float px, float py, float pz, float dx,
                        float fx, float fy, float fz, int snx, int sny, int snz, int ax,
                        float inv, float *vel_out, float *c_out) {
  int i0 = (int)floorf(fx), j0 = (int)floorf(fy), k0 = (int)floorf(fz);
  float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
  float acc = 0.0f, c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj)
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
        float val = f[((int64_t)ii * sny + jj) * snz + kk];
        float t = wt * val;
        acc = acc + t;
        float ox = ax == 0 ? (float)ii * dx - px : ((float)ii + 0.5f) * dx - px;
        float oy = ax == 1 ? (float)jj * dx - py : ((float)jj + 0.5f) * dx - py;
        float oz = ax == 2 ? (float)kk * dx - pz : ((float)kk + 0.5f) * dx - pz;
        float fu = t * inv;
        t = fu * ox; c0 = c0 + t;
        t = fu * oy; c1 = c1 + t;
        t = fu * oz; c2 = c2 + t;
      }
  *vel_out = acc;
  c_out[0] = c0; c_out[1] = c1; c_out[2] = c2;
}

/* k3_g2p_apic_advect, solver3d.py:1591-1732 */
void og_g2p_apic(int nx, int ny, int nz, float dx, float dt, const float *dom, int64_t P,
                 float *pos, float *vel, float *C, const float *u, const float *v,
                 const float *w, int par) {
#pragma omp parallel for schedule(static) if (par)
  for (int64_t pid = 0; pid < P; ++pid) {
    float px = pos[3 * pid], py = pos[3 * pid + 1], pz = pos[3 * pid + 2];
    float dd = dx * dx;
    float inv = 3.0f / dd;
    float gx = px / dx, gy = py / dx, gz = pz / dx;
    float hx = gx - 0.5f, hy = gy - 0.5f, hz = gz - 0.5f;
    float nu, nv, nw;
    apic_gather(u, px, py, pz, dx, gx - 0.0f, hy - 0.0f, hz - 0.0f, nx + 1, ny, nz, 0, inv,
                &nu, C + 9 * pid + 0);
    apic_gather(v, px, py, pz, dx, hx - 0.0f, gy - 0.0f, hz - 0.0f, nx, ny + 1, nz, 1, inv,
                &nv, C + 9 * pid + 3);
    apic_gather(w, px, py, pz, dx, hx - 0.0f, hy - 0.0f, gz - 0.0f, nx, ny, nz + 1, 2, inv,
                &nw, C + 9 * pid + 6);
    vel[3 * pid] = nu; vel[3 * pid + 1] = nv; vel[3 * pid + 2] = nw;
    advect(pos, pid, nu, nv, nw, dt, dx, dom);
  }
}

/* Canonical particle binning (new in this build; the reference has no sort):
 * key = tile-major cell index with 8x8x8 tiles; particles ordered by
 * (key, particle id).  Writes key[P], count[ntiles*512] and order[P] (the
 * storage index of the particle at each sorted slot).  pid gives each
 * particle's original id; stable counting sort over keys of particles
 * visited in pid order. */
void og_bin(int nx, int ny, int nz, float dx, int64_t P, const float *pos,
            const int32_t *pid, int32_t *key, int32_t *count, int64_t *order) {
  int ntx = (nx + 7) / 8, nty = (ny + 7) / 8, ntz = (nz + 7) / 8;
  int64_t nk = (int64_t)ntx * nty * ntz * 512;
  memset(count, 0, nk * 4);
  for (int64_t s = 0; s < P; ++s) {
    int ci = cell_of(pos[3 * s], dx, nx), cj = cell_of(pos[3 * s + 1], dx, ny),
        ck = cell_of(pos[3 * s + 2], dx, nz);
    int t = ((ci >> 3) * nty + (cj >> 3)) * ntz + (ck >> 3);
    key[s] = t * 512 + (((ci & 7) * 8 + (cj & 7)) * 8 + (ck & 7));
    count[key[s]]++;
  }
  int64_t *start = (int64_t *)malloc((nk + 1) * sizeof(int64_t));
  start[0] = 0;
  for (int64_t q = 0; q < nk; ++q) start[q + 1] = start[q] + count[q];
  /* visit storage slots in increasing pid order for a stable placement */
  int64_t *by_pid = (int64_t *)malloc((P > 0 ? P : 1) * sizeof(int64_t));
  for (int64_t s = 0; s < P; ++s) by_pid[pid[s]] = s;
  for (int64_t q = 0; q < P; ++q) {
    int64_t s = by_pid[q];
    order[start[key[s]]++] = s;
  }
  free(by_pid);
  free(start);
}

/* k_density_scatter, meshing/surface.py:14-43: cell-centred trilinear splat of
 * unit mass (the cfg4 loss operator). */
void og_density_splat(int nx, int ny, int nz, float dx, int64_t P, const float *pos,
                      float *rho_out) {
  memset(rho_out, 0, (int64_t)nx * ny * nz * 4);
  for (int64_t pid = 0; pid < P; ++pid) {
    float fx = pos[3 * pid] / dx - 0.5f, fy = pos[3 * pid + 1] / dx - 0.5f,
          fz = pos[3 * pid + 2] / dx - 0.5f;
    int i0 = (int)floorf(fx), j0 = (int)floorf(fy), k0 = (int)floorf(fz);
    float sx = fx - (float)i0, sy = fy - (float)j0, sz = fz - (float)k0;
    for (int di = 0; di < 2; ++di)
      for (int dj = 0; dj < 2; ++dj)
        for (int dk = 0; dk < 2; ++dk) {
          int ii = i0 + di, jj = j0 + dj, kk = k0 + dk;
          if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= nz) continue;
          float wx = di ? sx : 1.0f - sx, wy = dj ? sy : 1.0f - sy, wz = dk ? sz : 1.0f - sz;
          float wgt = wx * wy;
          wgt = wgt * wz;
          rho_out[CIDX(ii, jj, kk)] += wgt;
        }
  }
}
