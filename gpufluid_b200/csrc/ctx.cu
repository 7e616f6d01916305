// C ABI entry points of libgfb200: context lifecycle, binding, stage calls.
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

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

SegIndex seg_index(const Ctx *c) {
  const int64_t m = c->nseg + 1;
  return SegIndex{c->seg, c->seg_off, c->seg_off + m, c->seg_off + 2 * m, c->seg_off + 3 * m,
                  c->nseg};
}

static void destroy(Ctx *c) {
  if (!c) return;
  free_particles(c);
  void *ps[] = {c->count, c->start, c->scan_part, c->vmax_dev, c->adj_faces, c->adj_part,
                c->seg, c->seg_off, c->seg_state, c->seg_slot0, c->pcg_blk_job0,
                c->pcg_jobs, c->region_scratch};
  for (void *p : ps)
    if (p) cudaFree(p);
  if (c->seg_state_host) cudaFreeHost(c->seg_state_host);
  pressure_free(c);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  delete c;
}

// Device check and the allocations every context needs once its totals
// (ntiles, ncell, nkeys) are set.
static int new_ctx(Ctx **out) {
  *out = nullptr;
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
  *out = c;
  return GF_OK;
}

// Layout of a batch: scenes concatenated in table order.
static int plan_batch(const gf_grid_desc *scenes, int32_t n, gf_scene_layout *rows,
                      gf_batch_totals *tot) {
  if (!scenes || n < 1) return GF_INVALID_ARG;
  int64_t cell = 0, fu = 0, fv = 0, fw = 0, tile = 0, fslot = 0;
  for (int s = 0; s < n; ++s) {
    const gf_grid_desc &g = scenes[s];
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || !(g.dx > 0.f)) return GF_INVALID_ARG;
    const int64_t nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t nt = ((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8);
    if (rows) rows[s] = gf_scene_layout{cell, fu, fv, fw, tile, nt, fslot};
    cell += nx * ny * nz;
    fu += (nx + 1) * ny * nz;
    fv += nx * (ny + 1) * nz;
    fw += nx * ny * (nz + 1);
    tile += nt;
    fslot += (nx + 1) * (ny + 1) * (nz + 1);
  }
  if ((tile * 512) > INT32_MAX) return GF_INVALID_ARG;  // sort keys are int32
  if (tot) *tot = gf_batch_totals{cell, fu, fv, fw, tile, fslot};
  return GF_OK;
}


static int alloc_common(Ctx *c, int64_t max_particles) {
  c->nkeys = (int64_t)c->ntiles * gf::TILE_CELLS;
  c->n_scan_blocks = (c->nkeys + 4095) / 4096;
  int e;
  if ((e = check_cuda(c, cudaMalloc(&c->count, c->nkeys * 4), "alloc count")) ||
      (e = check_cuda(c, cudaMalloc(&c->start, (c->nkeys + 1) * 4), "alloc start")) ||
      (e = check_cuda(c, cudaMalloc(&c->scan_part, (c->n_scan_blocks + 1) * 4), "alloc scan")) ||
      (e = check_cuda(c, cudaMalloc(&c->vmax_dev, 16), "alloc vmax")) ||
      (e = pressure_alloc(c)) || (e = alloc_particles(c, max_particles)))
    return e;
  for (auto &ev : c->ev) cudaEventCreate(&ev);
  return GF_OK;
}

}  // namespace gf

using gf::Ctx;

static Ctx *as_ctx(void *p) { return reinterpret_cast<Ctx *>(p); }

extern "C" {

int gf_batch_plan(const gf_grid_desc *scenes, int32_t n, gf_scene_layout *rows,
                  gf_batch_totals *tot) {
  return gf::plan_batch(scenes, n, rows, tot);
}


int gf_batch_create(const gf_grid_desc *scenes, int32_t n, int64_t max_particles,
                    void **ctx_out) {
  if (!scenes || !ctx_out || n < 1 || max_particles < 0) return GF_INVALID_ARG;
  *ctx_out = nullptr;
  gf_batch_totals tot;
  std::vector<gf_scene_layout> lay(n);
  int e = gf::plan_batch(scenes, n, lay.data(), &tot);
  if (e) return e;
  Ctx *c = nullptr;
  if ((e = gf::new_ctx(&c))) return e;
  c->nseg = n;
  c->ntiles = (int)tot.ntiles;
  c->ncell = tot.ncell;
  c->nu = tot.nu; c->nv = tot.nv; c->nw = tot.nw;
  c->nfslot = tot.nslot;
  std::vector<gf::SegRow> rows(n);
  std::vector<int64_t> off(4 * (n + 1), 0);
  for (int s = 0; s < n; ++s) {
    const gf_grid_desc &g = scenes[s];
    gf::SegRow &r = rows[s];
    r.nx = g.nx; r.ny = g.ny; r.nz = g.nz;
    r.ntx = (g.nx + 7) / 8; r.nty = (g.ny + 7) / 8; r.ntz = (g.nz + 7) / 8;
    r.dx = g.dx; r.dom0 = g.dom[0]; r.dom1 = g.dom[1]; r.dom2 = g.dom[2];
    r.tile0 = lay[s].tile0; r.cell0 = lay[s].cell0;
    r.fu0 = lay[s].fu0; r.fv0 = lay[s].fv0; r.fw0 = lay[s].fw0; r.fslot0 = lay[s].fslot0;
    off[s] = lay[s].tile0;
    off[(n + 1) + s] = lay[s].cell0;
    off[2 * (n + 1) + s] = lay[s].fslot0;
  }
  off[n] = tot.ntiles;
  off[(n + 1) + n] = tot.ncell;
  off[2 * (n + 1) + n] = tot.nslot;
  // particle prefix: zeros until gf_batch_bind
  if ((e = gf::check_cuda(c, cudaMalloc(&c->seg, n * sizeof(gf::SegRow)), "alloc segments")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->seg_off, off.size() * 8), "alloc segment prefix")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->seg_state, n * sizeof(gf::PcgState)),
                          "alloc scene states")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->seg_slot0, (n + 1) * 4), "alloc scene slots")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->pcg_blk_job0, (gf::MAX_PCG_BLOCKS + 1) * 4),
                          "alloc PCG job ranges")) ||
      (e = gf::check_cuda(c, cudaMalloc(&c->pcg_jobs, gf::pcg_jobs_bytes(n)),
                          "alloc PCG jobs")) ||
      (e = gf::check_cuda(c, cudaMallocHost((void **)&c->seg_state_host,
                                            n * sizeof(gf::PcgState)),
                          "alloc pinned scene states")) ||
      (e = gf::check_cuda(c, cudaMemcpy(c->seg, rows.data(), n * sizeof(gf::SegRow),
                                        cudaMemcpyHostToDevice),
                          "upload segments")) ||
      (e = gf::check_cuda(c, cudaMemcpy(c->seg_off, off.data(), off.size() * 8,
                                        cudaMemcpyHostToDevice),
                          "upload segment prefix")) ||
      (e = gf::check_cuda(c, cudaMemset(c->seg_state, 0, n * sizeof(gf::PcgState)),
                          "zero scene states")) ||
      (e = gf::alloc_common(c, max_particles))) {
    gf::destroy(c);
    return e;
  }
  *ctx_out = c;
  return GF_OK;
}

int gf_batch_bind(void *ctx, const gf_fields *f, const gf_particles *p, const int64_t *counts) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c || !f || !p || !counts) return GF_INVALID_ARG;
  if (c->nseg < 1) return gf::fail(c, GF_INVALID_ARG, "gf_batch_bind: not a batch context");
  std::vector<int64_t> part0(c->nseg + 1, 0);
  for (int s = 0; s < c->nseg; ++s) {
    if (counts[s] < 0) return gf::fail(c, GF_INVALID_ARG, "gf_batch_bind: negative count");
    part0[s + 1] = part0[s] + counts[s];
  }
  if (part0[c->nseg] != p->n)
    return gf::fail(c, GF_INVALID_ARG, "gf_batch_bind: scene counts do not sum to n");
  int e = gf::check_cuda(c, cudaMemcpy(c->seg_off + 3 * (c->nseg + 1), part0.data(),
                                       part0.size() * 8, cudaMemcpyHostToDevice),
                         "upload particle prefix");
  if (e) return e;
  return gf_bind(ctx, f, p);
}

int gf_batch_pressure_stats(void *ctx, int32_t *iters, double *relres, int32_t *status) {
  Ctx *c = reinterpret_cast<Ctx *>(ctx);
  if (!c) return GF_INVALID_ARG;
  if (c->nseg < 1) return gf::fail(c, GF_INVALID_ARG, "not a batch context");
  const bool pcg = c->last_solver == GF_PCG || c->last_solver == GF_PCG_REFINED;
  if (!pcg) {
    for (int s = 0; s < c->nseg; ++s) {
      if (iters) iters[s] = c->last_iters;
      if (relres) relres[s] = -1.0;
      if (status) status[s] = GF_OK;
    }
    return GF_OK;
  }
  int e = gf::check_cuda(c, cudaMemcpyAsync(c->seg_state_host, c->seg_state,
                                            c->nseg * sizeof(gf::PcgState),
                                            cudaMemcpyDeviceToHost, c->stream),
                         "read scene states");
  if (!e) e = gf::check_cuda(c, cudaMemcpyAsync(c->state_host, c->state, sizeof(gf::PcgState),
                                                cudaMemcpyDeviceToHost, c->stream),
                             "read barrier state");
  if (!e) e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync");
  if (e) return e;
  for (int s = 0; s < c->nseg; ++s) {
    const gf::PcgState &S = c->seg_state_host[s];
    if (iters) iters[s] = S.iters;
    if (relres) {
      if (c->last_solver == GF_PCG_REFINED)
        relres[s] = S.b2 > 0 ? sqrt(S.r_true2 / S.b2) : 0.0;
      else
        relres[s] = S.r0 > 0 ? sqrt(S.rr / S.r0) : 0.0;
    }
    if (status) status[s] = c->state_host->error ? GF_TIMEOUT : S.status;
  }
  if (c->state_host->error) return gf::fail(c, GF_TIMEOUT, "PCG grid barrier timed out");
  return GF_OK;
}


int gf_create(const gf_grid_desc *g, int64_t max_particles, void **ctx_out) {
  if (!g || !ctx_out) return GF_INVALID_ARG;
  *ctx_out = nullptr;
  if (g->nx < 1 || g->ny < 1 || g->nz < 1 || !(g->dx > 0.f) || max_particles < 0)
    return GF_INVALID_ARG;
  Ctx *c = nullptr;
  int e = gf::new_ctx(&c);
  if (e) return e;
  c->nx = g->nx; c->ny = g->ny; c->nz = g->nz; c->dx = g->dx;
  for (int q = 0; q < 3; ++q) c->dom[q] = g->dom[q];
  c->ntx = (c->nx + 7) / 8; c->nty = (c->ny + 7) / 8; c->ntz = (c->nz + 7) / 8;
  c->ntiles = c->ntx * c->nty * c->ntz;
  c->ncell = (int64_t)c->nx * c->ny * c->nz;
  c->nu = (int64_t)(c->nx + 1) * c->ny * c->nz;
  c->nv = (int64_t)c->nx * (c->ny + 1) * c->nz;
  c->nw = (int64_t)c->nx * c->ny * (c->nz + 1);
  c->nfslot = (int64_t)(c->nx + 1) * (c->ny + 1) * (c->nz + 1);
  if ((e = gf::alloc_common(c, max_particles))) {
    gf::destroy(c);
    return e;
  }
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
  return gf::encode_face_maps(c);
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

// A captured substep: the instantiated graph and the kernels it launches.
struct GfGraph {
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;
};

int gf_graph_capture(void *ctx, const gf_step_params *prm, void **graph_out) {
  Ctx *c = as_ctx(ctx);
  if (!c || !prm || !graph_out) return GF_INVALID_ARG;
  *graph_out = nullptr;
  cudaStream_t st = c->stream;
  bool own = false;
  if (!st) {  // the legacy default stream cannot be captured: use a private one
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      return gf::fail(c, GF_CUDA_ERROR, "gf_graph_capture: stream creation failed");
    }
    own = true;
  }
  // everything the substep reads must be ready before the capture's first node
  int e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "gf_graph_capture sync");
  if (e) {
    if (own) cudaStreamDestroy(st);
    return e;
  }
  const bool timing = c->timing;
  const cudaStream_t saved = c->stream;
  c->timing = false;
  c->stream = st;
  const int64_t before = c->launches;
  e = gf::check_cuda(c, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal),
                     "gf_graph_capture begin");
  int step_e = e ? e : gf_step(ctx, prm);
  cudaGraph_t graph = nullptr;
  if (!e) {
    const cudaError_t ee = cudaStreamEndCapture(st, &graph);
    if (!step_e && ee != cudaSuccess) step_e = gf::check_cuda(c, ee, "gf_graph_capture end");
  }
  c->timing = timing;
  c->stream = saved;
  const int64_t captured = c->launches - before;
  c->launches = before;  // capturing ran nothing
  GfGraph *g = nullptr;
  if (!step_e && graph) {
    g = new GfGraph();
    g->launches = captured;
    step_e = gf::check_cuda(c, cudaGraphInstantiate(&g->exec, graph, 0),
                            "gf_graph_capture instantiate");
  }
  if (graph) cudaGraphDestroy(graph);
  if (own) cudaStreamDestroy(st);
  if (step_e) {
    cudaGetLastError();
    delete g;
    return step_e;
  }
  *graph_out = g;
  return GF_OK;
}

int gf_graph_replay(void *ctx, void *graph) {
  Ctx *c = as_ctx(ctx);
  GfGraph *g = reinterpret_cast<GfGraph *>(graph);
  if (!c || !g || !g->exec) return GF_INVALID_ARG;
  int e = gf::check_cuda(c, cudaGraphLaunch(g->exec, c->stream), "gf_graph_replay");
  if (!e) c->launches += g->launches;
  return e;
}

int gf_graph_destroy(void *graph) {
  GfGraph *g = reinterpret_cast<GfGraph *>(graph);
  if (!g) return GF_INVALID_ARG;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  delete g;
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
  info->coarse = (info->kernel != 0 && c->state_host->coarse_used) ? 1 : 0;
  return e;
}

int gf_bounds_status(int32_t reset, int64_t *violations, int32_t *first_line,
                     int32_t *checked) {
  if (!violations || !first_line || !checked) return GF_INVALID_ARG;
#ifdef GF_BOUNDS_CHECK
  *checked = 1;
#else
  *checked = 0;
#endif
  *violations = 0;
  *first_line = 0;
  int (*readers[])(unsigned long long *, int *, int) = {gf::bounds_read_bin,
                                                        gf::bounds_read_transfer,
                                                        gf::bounds_read_pressure};
  for (auto rd : readers) {
    unsigned long long h = 0;
    int line = 0;
    const int e = rd(&h, &line, reset);
    if (e) return e;
    if (h && !*violations) *first_line = line;
    *violations += (int64_t)h;
  }
  return GF_OK;
}

int gf_health_read(void *ctx, int32_t reset, gf_health *out) {
  Ctx *c = as_ctx(ctx);
  if (!c || !out) return GF_INVALID_ARG;
  int32_t h[8];
  int e = gf::check_cuda(c, cudaMemcpyAsync(h, c->health, sizeof(h), cudaMemcpyDeviceToHost,
                                            c->stream),
                         "read solve health");
  if (e) return e;
  if (reset && (e = gf::check_cuda(c, cudaMemsetAsync(c->health, 0, sizeof(h), c->stream),
                                   "reset solve health")))
    return e;
  if ((e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "sync"))) return e;
  static const int32_t by_severity[5] = {GF_OK, GF_NOT_CONVERGED, GF_BREAKDOWN, GF_NAN,
                                         GF_TIMEOUT};
  auto status_of = [&](int32_t sev) { return by_severity[sev < 0 ? 0 : (sev > 4 ? 4 : sev)]; };
  out->worst_status = status_of(h[0]);
  out->solves = h[1];
  out->not_converged = h[2];
  out->failed = h[3];
  out->last_status = status_of(h[4]);
  out->wait_timeouts = h[5];
  return GF_OK;
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
