// C ABI entry points of libgfb200: context lifecycle, binding, stage calls.
#include <cstring>
#include <new>

#include "gf_internal.cuh"

namespace gf {

int fail(Ctx *c, int status, const std::string &msg) {
  if (c) c->err = msg;
  return status;
}

int check_cuda(Ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return GF_OK;
  return fail(c, GF_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(Ctx *c, const char *what) {
  return check_cuda(c, cudaGetLastError(), what);
}

static void free_particles(Ctx *c) {
  void *ps[] = {c->key, c->rank, c->order, c->rec0, c->rec1, c->rec2, c->rec3};
  for (void *p : ps)
    if (p) cudaFree(p);
  c->key = c->rank = c->order = nullptr;
  c->rec0 = c->rec1 = c->rec2 = c->rec3 = nullptr;
  c->cap = 0;
}

static int alloc_particles(Ctx *c, int64_t n) {
  if (n <= c->cap) return GF_OK;
  free_particles(c);
  int64_t m = n > 0 ? n : 1;
  int e;
  void **p32[] = {(void **)&c->key, (void **)&c->rank, (void **)&c->order};
  for (void **p : p32)
    if ((e = check_cuda(c, cudaMalloc(p, m * 4), "alloc particle scratch"))) return e;
  void **p128[] = {(void **)&c->rec0, (void **)&c->rec1, (void **)&c->rec2, (void **)&c->rec3};
  for (void **p : p128)
    if ((e = check_cuda(c, cudaMalloc(p, m * 16), "alloc particle records"))) return e;
  c->cap = n;
  return GF_OK;
}

static void destroy(Ctx *c) {
  if (!c) return;
  free_particles(c);
  void *ps[] = {c->count, c->start, c->scan_part, c->vmax_dev, c->adj_faces, c->adj_part};
  for (void *p : ps)
    if (p) cudaFree(p);
  pressure_free(c);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  delete c;
}

}  // namespace gf

using gf::Ctx;

static Ctx *as_ctx(void *p) { return reinterpret_cast<Ctx *>(p); }

extern "C" {

int gf_create(const gf_grid_desc *g, int64_t max_particles, void **ctx_out) {
  if (!g || !ctx_out) return GF_INVALID_ARG;
  *ctx_out = nullptr;
  if (g->nx < 1 || g->ny < 1 || g->nz < 1 || !(g->dx > 0.f) || max_particles < 0)
    return GF_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return GF_NO_DEVICE;
  }
  Ctx *c = new (std::nothrow) Ctx();
  if (!c) return GF_CUDA_ERROR;
  cudaGetDevice(&c->device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess || prop.major < 10) {
    delete c;
    return GF_NO_DEVICE;
  }
  c->num_sms = prop.multiProcessorCount;
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz; c->dx = g->dx;
  for (int q = 0; q < 3; ++q) c->dom[q] = g->dom[q];
  c->ntx = (c->nx + 7) / 8; c->nty = (c->ny + 7) / 8; c->ntz = (c->nz + 7) / 8;
  c->ntiles = c->ntx * c->nty * c->ntz;
  c->nkeys = (int64_t)c->ntiles * gf::TILE_CELLS;
  c->ncell = (int64_t)c->nx * c->ny * c->nz;
  c->n_scan_blocks = (c->nkeys + 4095) / 4096;
  int e;
  if ((e = gf::check_cuda(c, cudaMalloc(&c->count, c->nkeys * 4), "alloc count")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->start, (c->nkeys + 1) * 4), "alloc start")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->scan_part, (c->n_scan_blocks + 1) * 4), "alloc scan")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->vmax_dev, 16), "alloc vmax")) ||
      (e = gf::pressure_alloc(c)) || (e = gf::alloc_particles(c, max_particles))) {
    gf::destroy(c);
    return e;
  }
  for (auto &ev : c->ev) cudaEventCreate(&ev);
  *ctx_out = c;
  return GF_OK;
}

int gf_destroy(void *ctx) {
  gf::destroy(as_ctx(ctx));
  return GF_OK;
}

int gf_reserve_particles(void *ctx, int64_t n) {
  Ctx *c = as_ctx(ctx);
  if (!c || n < 0) return GF_INVALID_ARG;
  if (n > INT32_MAX) return gf::fail(c, GF_INVALID_ARG, "particle count exceeds int32 range");
  return gf::alloc_particles(c, n);
}

int gf_bind(void *ctx, const gf_fields *f, const gf_particles *p) {
  Ctx *c = as_ctx(ctx);
  if (!c || !f || !p) return GF_INVALID_ARG;
  if (!f->u || !f->v || !f->w || !f->uw || !f->vw || !f->ww || !f->us || !f->vs || !f->ws ||
      !f->p || !f->div || !f->label)
    return gf::fail(c, GF_INVALID_ARG, "gf_bind: a required field pointer is NULL");
  if (reinterpret_cast<uintptr_t>(f->label) % 4)
    return gf::fail(c, GF_INVALID_ARG, "gf_bind: label must be 4-byte aligned");
  if (p->n < 0 || (p->n > 0 && (!p->pos || !p->vel || !p->pid)))
    return gf::fail(c, GF_INVALID_ARG, "gf_bind: particle buffers missing");
  int e = gf::alloc_particles(c, p->n);
  if (e) return e;
  c->f = *f;
  c->p = *p;
  c->bound = true;
  return GF_OK;
}

int gf_set_stream(void *ctx, void *stream) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  c->stream = reinterpret_cast<cudaStream_t>(stream);
  return GF_OK;
}

const char *gf_last_error(void *ctx) {
  Ctx *c = as_ctx(ctx);
  return c ? c->err.c_str() : "null context";
}

int64_t gf_launch_count(void *ctx) {
  Ctx *c = as_ctx(ctx);
  return c ? c->launches : 0;
}

int gf_bin(void *ctx, int32_t transfer) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  return gf::launch_bin(c, transfer);
}

int gf_p2g(void *ctx, int32_t transfer) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (transfer < GF_FLIP || transfer > GF_APIC) return gf::fail(c, GF_INVALID_ARG, "bad transfer");
  return gf::launch_p2g(c, transfer);
}

int gf_forces_div(void *ctx, float gravity, float dt, float rho) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (!(dt > 0.f)) return gf::fail(c, GF_INVALID_ARG, "dt must be > 0");
  return gf::launch_forces_div(c, gravity, dt, rho);
}

int gf_pressure(void *ctx, const gf_step_params *prm, int32_t *iters_out) {
  Ctx *c = as_ctx(ctx);
  if (!c || !prm) return GF_INVALID_ARG;
  int e = gf::launch_pressure(c, prm);
  if (e || !iters_out) return e;
  int32_t it;
  double rel;
  int32_t status;
  e = gf_pressure_result(ctx, &it, &rel, &status);
  *iters_out = it;
  return e;
}

int gf_project(void *ctx, float dt, float rho) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  return gf::launch_project(c, dt, rho);
}

int gf_g2p(void *ctx, int32_t transfer, float flip_blend, float dt) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (transfer < GF_FLIP || transfer > GF_APIC) return gf::fail(c, GF_INVALID_ARG, "bad transfer");
  return gf::launch_g2p(c, transfer, flip_blend, dt);
}

int gf_step(void *ctx, const gf_step_params *prm) {
  Ctx *c = as_ctx(ctx);
  if (!c || !prm) return GF_INVALID_ARG;
  if (prm->transfer < GF_FLIP || prm->transfer > GF_APIC)
    return gf::fail(c, GF_INVALID_ARG, "bad transfer");
  if (!(prm->dt > 0.f)) return gf::fail(c, GF_INVALID_ARG, "dt must be > 0");
  cudaStream_t st = c->stream;
  int e;
  if (c->timing) cudaEventRecord(c->ev[0], st);
  if ((e = gf::launch_bin(c, prm->transfer))) return e;
  if (c->timing) cudaEventRecord(c->ev[1], st);
  if ((e = gf::launch_p2g(c, prm->transfer))) return e;
  if (c->timing) cudaEventRecord(c->ev[2], st);
  if ((e = gf::launch_forces_div(c, prm->gravity, prm->dt, prm->rho))) return e;
  if (c->timing) cudaEventRecord(c->ev[3], st);
  if ((e = gf::launch_pressure(c, prm))) return e;
  if (c->timing) cudaEventRecord(c->ev[4], st);
  if ((e = gf::launch_project(c, prm->dt, prm->rho))) return e;
  if (c->timing) cudaEventRecord(c->ev[5], st);
  // the reference's PIC mode is the same kernel with the caller's flip_blend
  if ((e = gf::launch_g2p(c, prm->transfer, prm->flip_blend, prm->dt))) return e;
  if (c->timing) cudaEventRecord(c->ev[6], st);
  return GF_OK;
}

int gf_pressure_result(void *ctx, int32_t *iters, double *relres, int32_t *status) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (c->last_solver == GF_PCG || c->last_solver == GF_PCG_REFINED) {
    int e = gf::check_cuda(c, cudaMemcpyAsync(c->state_host, c->state, sizeof(gf::PcgState),
                                              cudaMemcpyDeviceToHost, c->stream),
                           "read pcg state");
    if (e) return e;
    if ((e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync"))) return e;
    const gf::PcgState &s = *c->state_host;
    if (iters) *iters = s.iters;
    if (relres) {
      if (c->last_solver == GF_PCG_REFINED)
        *relres = s.b2 > 0 ? sqrt(s.r_true2 / s.b2) : 0.0;
      else
        *relres = s.r0 > 0 ? sqrt(s.rr / s.r0) : 0.0;
    }
    if (status) *status = s.error ? GF_TIMEOUT : s.status;
    if (s.error) return gf::fail(c, GF_TIMEOUT, "PCG grid barrier timed out");
    return GF_OK;
  }
  if (iters) *iters = c->last_iters;
  if (relres) *relres = -1.0;
  if (status) *status = GF_OK;
  return GF_OK;
}

int gf_bin_read(void *ctx, int32_t *key, int32_t *count, int32_t *order, int64_t *nkeys) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (nkeys) *nkeys = c->nkeys;
  const int64_t n = c->bound ? c->p.n : 0;
  int e;
  struct { int32_t *dst; const int32_t *src; int64_t len; } cp[3] = {
      {key, c->key, n}, {count, c->count, c->nkeys}, {order, c->order, n}};
  for (auto &q : cp)
    if (q.dst && q.len > 0 &&
        (e = gf::check_cuda(c, cudaMemcpyAsync(q.dst, q.src, q.len * 4, cudaMemcpyDeviceToHost,
                                               c->stream), "gf_bin_read")))
      return e;
  return gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync");
}

int gf_enable_timing(void *ctx, int32_t on) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  c->timing = on != 0;
  return GF_OK;
}

int gf_stage_times(void *ctx, float *ms8) {
  Ctx *c = as_ctx(ctx);
  if (!c || !ms8) return GF_INVALID_ARG;
  if (!c->timing) return gf::fail(c, GF_INVALID_ARG, "timing is off");
  int e = gf::check_cuda(c, cudaEventSynchronize(c->ev[6]), "sync timing");
  if (e) return e;
  for (int q = 0; q < 6; ++q) cudaEventElapsedTime(&ms8[q], c->ev[q], c->ev[q + 1]);
  cudaEventElapsedTime(&ms8[6], c->ev[0], c->ev[6]);
  cudaEventElapsedTime(&ms8[7], c->ev[8], c->ev[9]);
  return GF_OK;
}

int gf_pcg_trace(void *ctx, int64_t *host, int32_t cap, int32_t *n) {
  Ctx *c = as_ctx(ctx);
  if (!c || !n) return GF_INVALID_ARG;
  int32_t it;
  double rel;
  int32_t status;
  int e = gf_pressure_result(ctx, &it, &rel, &status);
  if (e) return e;
  int32_t cnt = c->state_host->trace_n;
  *n = cnt;
  if (host && cap > 0) {
    // block 0's stamps fill the first half, per-block (busy cycles, tiles)
    // pairs the second half of the buffer
    int32_t m = cap < gf::TRACE_CAP ? cap : gf::TRACE_CAP;
    if (m > 0 && (e = gf::check_cuda(c, cudaMemcpy(host, c->trace, (size_t)m * 8,
                                                   cudaMemcpyDeviceToHost), "read trace")))
      return e;
  }
  return GF_OK;
}

int gf_pressure_stats(void *ctx, gf_pressure_info *info) {
  Ctx *c = as_ctx(ctx);
  if (!c || !info) return GF_INVALID_ARG;
  int32_t it = 0, status = 0;
  double rel = -1.0;
  int e = gf_pressure_result(ctx, &it, &rel, &status);
  if (e && e != GF_TIMEOUT) return e;
  int32_t host[4] = {0, 0, 0, 0};
  int e2 = gf::check_cuda(c, cudaMemcpy(host, c->n_active, 16, cudaMemcpyDeviceToHost),
                          "read active/fluid counts");
  if (e2) return e2;
  info->iters = it;
  info->status = status;
  info->relres = rel;
  info->n_active_tiles = host[0];
  int64_t nf;
  memcpy(&nf, &host[2], 8);
  info->n_fluid = nf;
  info->replacements = (c->last_solver == GF_PCG_REFINED) ? c->state_host->n_replace : 0;
  info->kernel = 0;
  if (c->last_solver == GF_PCG || c->last_solver == GF_PCG_REFINED)
    info->kernel = c->state_host->smem_solver ? 1 : 2;
  info->pad = 0;
  return e;
}

int gf_active_tiles(void *ctx, int32_t *n_active, const int32_t **tiles) {
  Ctx *c = as_ctx(ctx);
  if (!c) return GF_INVALID_ARG;
  if (n_active) {
    int e = gf::check_cuda(c, cudaMemcpyAsync(n_active, c->n_active, 4, cudaMemcpyDeviceToHost,
                                              c->stream), "read n_active");
    if (e) return e;
    if ((e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync"))) return e;
  }
  if (tiles) *tiles = c->tile_list;
  return GF_OK;
}

int gf_vmax(void *ctx, float *vmax_out) {
  Ctx *c = as_ctx(ctx);
  if (!c || !vmax_out) return GF_INVALID_ARG;
  int e = gf::launch_vmax(c);
  if (e) return e;
  float v2 = 0.f;
  if ((e = gf::check_cuda(c, cudaMemcpyAsync(&v2, c->vmax_dev, 4, cudaMemcpyDeviceToHost,
                                             c->stream), "read vmax")))
    return e;
  if ((e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync"))) return e;
  *vmax_out = sqrtf(v2);
  return GF_OK;
}

}  // extern "C"
