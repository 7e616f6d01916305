// Launch-shape autotuner.
//
// gf_autotune times real substeps of the bound scene (or batch) with the
// stage events of gf_step and picks, one knob after the other (coordinate
// descent), the fastest of a few candidates:
//   p2g_tiles_k, g2p_tiles_k    tile shape of P2G and of the tile-staged G2P
//                               (single grid): blocks of 8 x 8 x 8 cells (1)
//                               or 8 x 8 x 16 (2); for G2P also 0, the
//                               unstaged per-particle kernel   (P2G, G2P stage)
//   p2g_map                     P2G lanes: runs of particles (0), one cell
//                               each (1), one cell each summed in registers
//                               first (2), the same from coalesced shared
//                               staging (3) or from warp-staged rounds of 8
//                               (4) or 4 (5) particles per cell  (P2G stage)
//   g2p_threads                 threads per block of the batches' per-particle
//                               G2P                                 (G2P stage)
//   grid_threads, blocks_per_sm launch shape of the grid-stride face/cell
//                               kernels (forces, divergence, project)
//   pcg_blocks_per_sm           resident blocks per SM of the global-memory
//                               (and segmented) PCG; 0 = occupancy maximum
// Every trial starts from the same particle state (snapshotted on entry and
// restored before each trial and on exit), so tuning leaves the simulation
// where it was.  The chosen shapes stay in the context; gf_get_tune /
// gf_set_tune read or impose them (a host cache can replay a choice).
#include <vector>

#include "gf_internal.cuh"

namespace gf {

struct Snapshot {
  float *pos = nullptr, *vel = nullptr, *C = nullptr;
  int32_t *pid = nullptr;
  int64_t n = 0;
};

static int snap_take(Ctx *c, Snapshot &s) {
  s.n = c->p.n;
  if (s.n == 0) return GF_OK;
  int e;
  if ((e = check_cuda(c, cudaMalloc(&s.pos, s.n * 12), "tune snapshot")) ||
      (e = check_cuda(c, cudaMalloc(&s.vel, s.n * 12), "tune snapshot")) ||
      (e = check_cuda(c, cudaMalloc(&s.pid, s.n * 4), "tune snapshot")))
    return e;
  if (c->p.C && (e = check_cuda(c, cudaMalloc(&s.C, s.n * 36), "tune snapshot"))) return e;
  cudaStream_t st = c->stream;
  if ((e = check_cuda(c, cudaMemcpyAsync(s.pos, c->p.pos, s.n * 12, cudaMemcpyDeviceToDevice, st),
                      "tune snapshot copy")) ||
      (e = check_cuda(c, cudaMemcpyAsync(s.vel, c->p.vel, s.n * 12, cudaMemcpyDeviceToDevice, st),
                      "tune snapshot copy")) ||
      (e = check_cuda(c, cudaMemcpyAsync(s.pid, c->p.pid, s.n * 4, cudaMemcpyDeviceToDevice, st),
                      "tune snapshot copy")))
    return e;
  if (s.C && (e = check_cuda(c, cudaMemcpyAsync(s.C, c->p.C, s.n * 36, cudaMemcpyDeviceToDevice, st),
                             "tune snapshot copy")))
    return e;
  return GF_OK;
}

static int snap_restore(Ctx *c, const Snapshot &s) {
  if (s.n == 0) return GF_OK;
  cudaStream_t st = c->stream;
  int e;
  if ((e = check_cuda(c, cudaMemcpyAsync(c->p.pos, s.pos, s.n * 12, cudaMemcpyDeviceToDevice, st),
                      "tune restore")) ||
      (e = check_cuda(c, cudaMemcpyAsync(c->p.vel, s.vel, s.n * 12, cudaMemcpyDeviceToDevice, st),
                      "tune restore")) ||
      (e = check_cuda(c, cudaMemcpyAsync(c->p.pid, s.pid, s.n * 4, cudaMemcpyDeviceToDevice, st),
                      "tune restore")))
    return e;
  if (s.C && (e = check_cuda(c, cudaMemcpyAsync(c->p.C, s.C, s.n * 36, cudaMemcpyDeviceToDevice, st),
                             "tune restore")))
    return e;
  return GF_OK;
}

static void snap_free(Snapshot &s) {
  void *ps[] = {s.pos, s.vel, s.C, s.pid};
  for (void *p : ps)
    if (p) cudaFree(p);
  s = Snapshot{};
}

// Stage times of one substep from the snapshot: [0] whole step, [1] G2P,
// [2] forces + divergence + project, [3] pressure solver kernel(s), [4] P2G.
static int trial(Ctx *c, const Snapshot &s, const gf_step_params *prm, float out[5]) {
  int e = snap_restore(c, s);
  if (e) return e;
  if ((e = gf_step(c, prm))) return e;
  if ((e = check_cuda(c, cudaStreamSynchronize(c->stream), "tune sync"))) return e;
  float t = 0.f;
  cudaEventElapsedTime(&out[0], c->ev[0], c->ev[6]);
  cudaEventElapsedTime(&out[1], c->ev[5], c->ev[6]);
  cudaEventElapsedTime(&t, c->ev[2], c->ev[3]);
  out[2] = t;
  cudaEventElapsedTime(&t, c->ev[4], c->ev[5]);
  out[2] += t;
  out[3] = 0.f;
  if (prm->solver == GF_PCG || prm->solver == GF_PCG_REFINED)
    cudaEventElapsedTime(&out[3], c->ev[8], c->ev[9]);
  cudaEventElapsedTime(&out[4], c->ev[1], c->ev[2]);
  return GF_OK;
}

// Best of `reps` trials of stage `which`.
static int measure(Ctx *c, const Snapshot &s, const gf_step_params *prm, int which, int reps,
                   float *best) {
  *best = 3.4e38f;
  for (int r = 0; r < reps; ++r) {
    float t[5];
    int e = trial(c, s, prm, t);
    if (e) return e;
    if (t[which] < *best) *best = t[which];
  }
  return GF_OK;
}

static void to_info(const Tune &t, gf_tune_info *o) {
  o->p2g_tiles_k = t.p2g_tiles_k;
  o->p2g_map = t.p2g_map;
  o->g2p_tiles_k = t.g2p_tiles_k;
  o->g2p_threads = t.g2p_threads;
  o->grid_threads = t.grid_threads;
  o->grid_blocks_per_sm = t.grid_blocks_per_sm;
  o->pcg_blocks_per_sm = t.pcg_blocks_per_sm;
}

}  // namespace gf

extern "C" {

int gf_autotune(void *ctx, const gf_step_params *prm, gf_tune_info *out) {
  gf::Ctx *c = reinterpret_cast<gf::Ctx *>(ctx);
  if (!c || !prm) return GF_INVALID_ARG;
  if (!c->bound) return gf::fail(c, GF_INVALID_ARG, "gf_autotune: buffers not bound");
  const bool was_timing = c->timing;
  c->timing = true;
  gf::Snapshot snap;
  int e = gf::snap_take(c, snap);
  float before = 0.f, after = 0.f;
  const int reps = 2;
  if (!e) e = gf::measure(c, snap, prm, 0, reps, &before);
  // tile shapes of P2G and G2P (single grid) and the P2G lane map (single
  // grid and batches), fastest stage time of each
  if (!e) {
    for (int knob = 0; knob < 3 && !e; ++knob) {
      if (c->nseg > 0 && knob != 1) continue;  // batches: 8^3 P2G tiles, per-particle G2P
      int &v = knob == 0 ? c->tune.p2g_tiles_k : (knob == 1 ? c->tune.p2g_map : c->tune.g2p_tiles_k);
      // P2G blocks 1..2 tiles, lane maps 0..5, G2P 0 (unstaged) ..2 tiles
      const int lo = knob == 0 ? 1 : 0, hi = knob == 1 ? 5 : 2;
      int best_v = v;
      float best = 3.4e38f;
      for (int x = lo; x <= hi; ++x) {
        v = x;
        float t;
        if ((e = gf::measure(c, snap, prm, knob == 2 ? 1 : 4, reps, &t))) break;
        if (t < best) { best = t; best_v = x; }
      }
      v = best_v;
    }
  }
  // G2P block size of the batches' per-particle kernel
  if (!e && c->nseg > 0) {
    const int cand[] = {128, 256, 512};
    int best_v = c->tune.g2p_threads;
    float best = 3.4e38f;
    for (int v : cand) {
      c->tune.g2p_threads = v;
      float t;
      if ((e = gf::measure(c, snap, prm, 1, reps, &t))) break;
      if (t < best) { best = t; best_v = v; }
    }
    c->tune.g2p_threads = best_v;
  }
  // grid-stride kernels: threads x resident-block cap
  if (!e) {
    const int cand[][2] = {{256, 16}, {256, 8}, {512, 8}, {512, 4}, {128, 32}};
    gf::Tune keep = c->tune;
    float best = 3.4e38f;
    for (auto &v : cand) {
      c->tune.grid_threads = v[0];
      c->tune.grid_blocks_per_sm = v[1];
      float t;
      if ((e = gf::measure(c, snap, prm, 2, reps, &t))) break;
      if (t < best) {
        best = t;
        keep.grid_threads = v[0];
        keep.grid_blocks_per_sm = v[1];
      }
    }
    c->tune.grid_threads = keep.grid_threads;
    c->tune.grid_blocks_per_sm = keep.grid_blocks_per_sm;
  }
  // global-memory PCG residency (used by batches and by regions too large
  // for the shared-memory solver)
  const bool pcg = prm->solver == GF_PCG || prm->solver == GF_PCG_REFINED;
  if (!e && pcg && (c->nseg > 0 || (prm->flags & GF_FLAG_GLOBAL_PCG) ||
                    !gf::pcg_smem_fits(c, prm->solver == GF_PCG_REFINED))) {
    const int cand[] = {0, 1, 2};
    int best_v = c->tune.pcg_blocks_per_sm;
    float best = 3.4e38f;
    for (int v : cand) {
      c->tune.pcg_blocks_per_sm = v;
      float t;
      if ((e = gf::measure(c, snap, prm, 3, reps, &t))) break;
      if (t < best) { best = t; best_v = v; }
    }
    c->tune.pcg_blocks_per_sm = best_v;
  }
  if (!e) e = gf::measure(c, snap, prm, 0, reps, &after);
  if (!e) e = gf::snap_restore(c, snap);
  if (!e) e = gf::check_cuda(c, cudaStreamSynchronize(c->stream), "tune sync");
  gf::snap_free(snap);
  c->timing = was_timing;
  if (out) {
    gf::to_info(c->tune, out);
    out->step_ms_before = before;
    out->step_ms_after = after;
  }
  return e;
}

int gf_get_tune(void *ctx, gf_tune_info *out) {
  gf::Ctx *c = reinterpret_cast<gf::Ctx *>(ctx);
  if (!c || !out) return GF_INVALID_ARG;
  gf::to_info(c->tune, out);
  out->step_ms_before = out->step_ms_after = 0.f;
  return GF_OK;
}

int gf_set_tune(void *ctx, const gf_tune_info *in) {
  gf::Ctx *c = reinterpret_cast<gf::Ctx *>(ctx);
  if (!c || !in) return GF_INVALID_ARG;
  auto ok_threads = [](int t, int hi) { return t >= 32 && t <= hi && t % 32 == 0; };
  if (!ok_threads(in->g2p_threads, 512) || !ok_threads(in->grid_threads, 1024) ||
      in->grid_blocks_per_sm < 1 || in->grid_blocks_per_sm > 64 || in->pcg_blocks_per_sm < 0 ||
      in->pcg_blocks_per_sm > 8 || in->p2g_tiles_k < 1 || in->p2g_tiles_k > 2 ||
      in->g2p_tiles_k < 0 || in->g2p_tiles_k > 2 || in->p2g_map < 0 || in->p2g_map > 5)
    return gf::fail(c, GF_INVALID_ARG, "gf_set_tune: launch shape out of range");
  c->tune.p2g_tiles_k = in->p2g_tiles_k;
  c->tune.p2g_map = in->p2g_map;
  c->tune.g2p_tiles_k = in->g2p_tiles_k;
  c->tune.g2p_threads = in->g2p_threads;
  c->tune.grid_threads = in->grid_threads;
  c->tune.grid_blocks_per_sm = in->grid_blocks_per_sm;
  c->tune.pcg_blocks_per_sm = in->pcg_blocks_per_sm;
  return GF_OK;
}

}  // extern "C"
