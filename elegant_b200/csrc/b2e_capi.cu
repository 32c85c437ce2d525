/*
 * C-ABI implementation (include/elegant_b200.h): context, device buffers and
 * the pass/element orchestration that replaces do_tracking's loop
 * (do_tracking.c:488-2640) for the supported subset.
 *
 * Orchestration of one b2e_track call:
 *   pass 0 is cut before every RFCA whose fiducial is not yet known; between
 *   the pieces a one-thread-per-instance kernel forms the Kahan mean arrival
 *   time (findFiducialTime, simple_rfca.c:62-262) on the particles that reach
 *   the cavity; everything after the last fiducial runs as fused multi-pass
 *   launches (passes_per_launch passes each, all by default).
 *   CSR elements (CSRCSBEND/CSRDRIFT) are collective and are executed by the
 *   CSR driver (b2e_csr.cu) between ring launches.
 */
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <vector>
#include <algorithm>
#include "b2e_lattice.h"
#include "b2e_csr.h"
#include "b2e_kernels.h"
#include "b2e_wakenet.h"



using namespace b2e;

static const int kTileThreads = 128;

template <typename T> struct DevBuf {
  T *ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap && ptr)
      return cudaSuccess;
    if (ptr)
      cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    bytes = (bytes + 255) & ~(size_t)255;
    cudaError_t e = cudaMalloc(&ptr, bytes);
    if (e == cudaSuccess)
      cap = bytes / sizeof(T);
    return e;
  }
  void release() {
    if (ptr)
      cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

struct b2e_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  /* lattice */
  std::vector<b2e_element> base;
  b2e_run_options opt{};
  bool lattice_loaded = false;
  CompiledLattice lat;            /* instance 0 / base */
  int n_inst = 1;
  std::vector<int64_t> inst_offsets{0, 0};
  std::vector<DevElem> elems_all; /* [n_inst][n_elems] */
  std::vector<DevRad> rads_all;   /* [n_inst][n_elems] */
  DevBuf<DevRad> d_rads;
  std::vector<DevAperture> aps_all;
  DevBuf<DevElem> d_elems;
  DevBuf<DevAperture> d_aps;
  DevBuf<DevRfState> d_rf;
  DevBuf<DevTile> d_tiles;
  DevBuf<int64_t> d_inst_offsets;
  std::vector<DevTile> tiles;
  /* particles */
  int64_t n = 0;
  DevBuf<double> d_cols[6];
  DevBuf<int64_t> d_ids;
  DevBuf<int32_t> d_lost_pass, d_lost_elem;
  DevBuf<unsigned int> d_flag;
  DevBuf<unsigned long long> d_counters;
  bool particles_loaded = false;
  /* external (device) particle pointers for b2e_track_device */
  DevParticles ext{};
  bool use_ext = false;
  bool radiates = false; /* some element of some instance reads the DevRad table (any_radiation) */
  CsrState csr;
  int pass_counter = 0; /* next pass to track in the current run */
  int64_t launches = 0; /* kernels launched by this context */
  /* autotuning of the ring-kernel occupancy variant */
  int tuned_variant = 0;
  std::vector<float> tune_ms;
  DevBuf<double> d_scratch;       /* 6 columns, for timing variants off the real state */
  DevBuf<int32_t> d_scratch_loss; /* 2 columns */
  /* ensemble history */
  std::vector<int> tile_first;     /* first tile of each instance, n_inst + 1 entries */
  DevBuf<int> d_tile_first;
  DevBuf<double> d_hist_partials;  /* [n_tiles][passes of the call][11] */
  DevBuf<double> d_hist_out;       /* [n_inst][passes of the call][5] */
  std::vector<double> history;     /* [pass][inst][5]: survivors, <x>, <y>, ex, ey */
  int hist_pass0 = 0, hist_passes = 0;
  DevBuf<double> d_tbt;      /* [tbt_records][4][n] */
  int tbt_records = 0;
  int64_t tbt_rows = 0;
  DevBuf<double> d_naff;     /* [4][3][n] NAFF results, then [4][n] tunes */
  DevBuf<int> d_naff_bad;
  /* lost-particle compaction: second set of particle buffers, survivors per instance */
  DevBuf<double> d_cmp_cols[6];
  DevBuf<int64_t> d_cmp_ids;
  DevBuf<int32_t> d_cmp_lost_pass, d_cmp_lost_elem;
  DevBuf<int> d_alive_inst;
  /* WATCH recording (b2e_set_watch): [records][7][watch_rows] of the last call */
  int64_t watch_max_bytes = 0;
  DevBuf<double> d_watch;
  std::vector<int64_t> watch_rec0;   /* per WATCH ordinal: record of its first pass in the call */
  std::vector<int32_t> watch_first;  /* per WATCH ordinal: first pass it records in the call, -1: none */
  std::vector<int32_t> watch_rec_elem, watch_rec_pass;
  int64_t watch_rows = 0;
  bool watch_on = false;
};

static int fail(b2e_ctx *ctx, int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx)
    ctx->err = buf;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                                     \
  do {                                                                                                           \
    cudaError_t e_ = (call);                                                                                     \
    if (e_ != cudaSuccess)                                                                                       \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? B2E_ERR_NOMEM : B2E_ERR_CUDA, "%s: %s (%s:%d)", #call, \
                  cudaGetErrorString(e_), __FILE__, __LINE__);                                                   \
  } while (0)

extern "C" int b2e_version(void) { return 1; }

extern "C" int b2e_create(b2e_ctx **out, int device) {
  if (!out)
    return B2E_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= 0)
    return B2E_ERR_CUDA;
  if (device < 0 || device >= ndev)
    return B2E_ERR_ARG;
  b2e_ctx *ctx = new b2e_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return B2E_ERR_CUDA;
  }
  *out = ctx;
  return B2E_OK;
}

extern "C" int b2e_destroy(b2e_ctx *ctx) {
  if (!ctx)
    return B2E_ERR_ARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->d_elems.release();
  ctx->d_rads.release();
  ctx->d_tbt.release();
  ctx->d_naff.release();
  ctx->d_naff_bad.release();
  ctx->d_aps.release();
  ctx->d_rf.release();
  ctx->d_tiles.release();
  ctx->d_inst_offsets.release();
  for (auto &c : ctx->d_cols)
    c.release();
  ctx->d_ids.release();
  ctx->d_lost_pass.release();
  ctx->d_lost_elem.release();
  ctx->d_flag.release();
  ctx->d_counters.release();
  for (auto &c : ctx->d_cmp_cols)
    c.release();
  ctx->d_cmp_ids.release();
  ctx->d_cmp_lost_pass.release();
  ctx->d_cmp_lost_elem.release();
  ctx->d_alive_inst.release();
  csr_release(ctx->csr);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return B2E_OK;
}

extern "C" const char *b2e_last_error(const b2e_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" void *b2e_stream(b2e_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" int64_t b2e_kernel_launches(const b2e_ctx *ctx) { return ctx ? ctx->launches : -1; }

extern "C" int b2e_ring_tuning(const b2e_ctx *ctx, int32_t *chosen, float *ms_per_variant) {
  if (!ctx || !chosen)
    return B2E_ERR_ARG;
  *chosen = ctx->opt.ring_variant >= 1 && ctx->opt.ring_variant <= B2E_RING_VARIANTS ? ctx->opt.ring_variant
                                                                                     : ctx->tuned_variant;
  if (ms_per_variant)
    for (int v = 0; v < B2E_RING_VARIANTS; v++)
      ms_per_variant[v] = v < (int)ctx->tune_ms.size() ? ctx->tune_ms[v] : 0.f;
  return B2E_OK;
}

/* Rebuild the tile table for the current instance partition (every particle
 * of instance i, or its first alive[i] after a compaction). */
static void build_tiles(b2e_ctx *ctx, const int *alive = nullptr) {
  ctx->tiles.clear();
  ctx->tile_first.assign(1, 0);
  for (int i = 0; i < ctx->n_inst; i++) {
    const int64_t end = alive ? ctx->inst_offsets[i] + alive[i] : ctx->inst_offsets[i + 1];
    for (int64_t s = ctx->inst_offsets[i]; s < end; s += kTileThreads) {
      DevTile t;
      t.start = s;
      t.count = (int32_t)std::min<int64_t>(kTileThreads, end - s);
      t.inst = i;
      ctx->tiles.push_back(t);
    }
    ctx->tile_first.push_back((int)ctx->tiles.size());
  }
}

static int upload_tiles(b2e_ctx *ctx) {
  CUDA_TRY(ctx, ctx->d_tiles.ensure(std::max<size_t>(ctx->tiles.size(), 1)));
  if (!ctx->tiles.empty())
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_tiles.ptr, ctx->tiles.data(), sizeof(DevTile) * ctx->tiles.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
  return B2E_OK;
}

static int upload_lattice_tables(b2e_ctx *ctx) {
  CUDA_TRY(ctx, ctx->d_rads.ensure(ctx->rads_all.size()));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_rads.ptr, ctx->rads_all.data(), sizeof(DevRad) * ctx->rads_all.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, ctx->d_elems.ensure(ctx->elems_all.size()));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_elems.ptr, ctx->elems_all.data(), sizeof(DevElem) * ctx->elems_all.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, ctx->d_aps.ensure(std::max<size_t>(ctx->aps_all.size(), 1)));
  if (!ctx->aps_all.empty())
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_aps.ptr, ctx->aps_all.data(), sizeof(DevAperture) * ctx->aps_all.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, ctx->d_rf.ensure(std::max<size_t>((size_t)ctx->n_inst * ctx->lat.n_rf, 1)));
  CUDA_TRY(ctx, ctx->d_inst_offsets.ensure(ctx->inst_offsets.size()));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_inst_offsets.ptr, ctx->inst_offsets.data(),
                                sizeof(int64_t) * ctx->inst_offsets.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, ctx->d_tile_first.ensure(ctx->tile_first.size()));
  CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_tile_first.ptr, ctx->tile_first.data(), sizeof(int) * ctx->tile_first.size(),
                                cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, ctx->d_tiles.ensure(std::max<size_t>(ctx->tiles.size(), 1)));
  if (!ctx->tiles.empty())
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_tiles.ptr, ctx->tiles.data(), sizeof(DevTile) * ctx->tiles.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return B2E_OK;
}

/* the lattice needs the ring kernel's RAD instantiation: some element
 * radiates, steers (KQUAD/KSEXT HKICK/VKICK), is a KQUAD with fringe fields,
 * or is a bend with field terms, ETILT or second-order edges (all read the
 * DevRad table) */
static bool any_radiation(const std::vector<DevElem> &elems) {
  for (const DevElem &d : elems)
    if (d.flags & (EF_SR | EF_ISR | EF_FIELD | EF_ETILT | EF_EDGE_ORDER2 | EF_STEERING | EF_QFRINGE1 | EF_QFRINGE2 | \
                   EF_END_DRIFT | EF_EDGE1_SIMPLE | EF_EDGE2_SIMPLE))
      return true;
  return false;
}

extern "C" int b2e_element_defaults(int32_t type, b2e_element *element) {
  if (!element || type < B2E_DRIF || type > B2E_WATCH)
    return B2E_ERR_ARG;
  element->type = type;
  element->reserved = 0;
  b2e::element_defaults(type, element->p);
  return B2E_OK;
}

extern "C" int b2e_load_lattice(b2e_ctx *ctx, const b2e_element *elements, int32_t n_elements,
                                const b2e_run_options *options) {
  if (!ctx || !elements || n_elements <= 0 || !options)
    return fail(ctx, B2E_ERR_ARG, "b2e_load_lattice: null argument or empty lattice");
  if (options->p_central <= 0)
    return fail(ctx, B2E_ERR_ARG, "b2e_load_lattice: p_central must be positive");
  if (options->n_passes < 0)
    return fail(ctx, B2E_ERR_ARG, "b2e_load_lattice: n_passes must be >= 0");
  cudaSetDevice(ctx->device);
  ctx->opt = *options;
  if (ctx->opt.default_order <= 0)
    ctx->opt.default_order = 2;
  if (ctx->opt.coord_limit <= 0)
    ctx->opt.coord_limit = 10;
  if (ctx->opt.slope_limit <= 0)
    ctx->opt.slope_limit = 1;
  std::string e = compile_lattice(elements, n_elements, ctx->opt, ctx->lat);
  if (!e.empty())
    return fail(ctx, B2E_ERR_LATTICE, "%s", e.c_str());
  ctx->base.assign(elements, elements + n_elements);
  ctx->n_inst = 1;
  ctx->inst_offsets = {0, ctx->n};
  ctx->elems_all = ctx->lat.elems;
  ctx->rads_all = ctx->lat.rads;
  ctx->aps_all = ctx->lat.aps;
  ctx->radiates = any_radiation(ctx->elems_all);
  build_tiles(ctx);
  ctx->lattice_loaded = true;
  int rc = csr_configure(ctx->csr, ctx->base.data(), n_elements, ctx->lat, ctx->opt, ctx->err);
  if (rc)
    return rc;
  return upload_lattice_tables(ctx);
}

extern "C" int b2e_load_ensemble(b2e_ctx *ctx, int32_t n_instances, const int64_t *offsets,
                                 const b2e_override *overrides, int32_t n_overrides) {
  if (!ctx || n_instances <= 0 || !offsets || (n_overrides > 0 && !overrides))
    return fail(ctx, B2E_ERR_ARG, "b2e_load_ensemble: bad arguments");
  if (!ctx->lattice_loaded)
    return fail(ctx, B2E_ERR_STATE, "b2e_load_ensemble: load a lattice first");
  for (int i = 0; i < n_instances; i++)
    if (offsets[i + 1] < offsets[i] || offsets[0] != 0)
      return fail(ctx, B2E_ERR_ARG, "b2e_load_ensemble: offsets must start at 0 and be nondecreasing");
  const int ne = (int)ctx->base.size();
  for (int k = 0; k < n_overrides; k++)
    if (overrides[k].element < 0 || overrides[k].element >= ne || overrides[k].slot < 0 ||
        overrides[k].slot >= B2E_MAX_PARAMS || !overrides[k].values)
      return fail(ctx, B2E_ERR_ARG, "b2e_load_ensemble: override %d out of range", k);
  for (int k = 0; k < n_overrides; k++) {
    const int t = ctx->base[overrides[k].element].type;
    if (t == B2E_CSRCSBEND || t == B2E_CSRDRIFT)
      return fail(ctx, B2E_ERR_LATTICE,
                  "b2e_load_ensemble: CSR elements are shared by all bunches and take no per-instance overrides");
    if (t == B2E_WATCH)
      return fail(ctx, B2E_ERR_LATTICE,
                  "b2e_load_ensemble: WATCH elements record every instance alike and take no per-instance overrides");
  }
  ctx->n_inst = n_instances;
  ctx->inst_offsets.assign(offsets, offsets + n_instances + 1);
  ctx->elems_all.clear();
  ctx->rads_all.clear();
  ctx->aps_all.clear();
  std::vector<b2e_element> inst(ctx->base);
  CompiledLattice cl;
  for (int i = 0; i < n_instances; i++) {
    inst = ctx->base;
    for (int k = 0; k < n_overrides; k++)
      inst[overrides[k].element].p[overrides[k].slot] = overrides[k].values[i];
    std::string e = compile_lattice(inst.data(), ne, ctx->opt, cl);
    if (!e.empty())
      return fail(ctx, B2E_ERR_LATTICE, "instance %d: %s", i, e.c_str());
    ctx->elems_all.insert(ctx->elems_all.end(), cl.elems.begin(), cl.elems.end());
    ctx->rads_all.insert(ctx->rads_all.end(), cl.rads.begin(), cl.rads.end());
    ctx->aps_all.insert(ctx->aps_all.end(), cl.aps.begin(), cl.aps.end());
  }
  ctx->radiates = any_radiation(ctx->elems_all);
  build_tiles(ctx);
  int rc = upload_lattice_tables(ctx);
  if (rc)
    return rc;
  if (ctx->csr.enabled && csr_set_bunches(ctx->csr, n_instances, ctx->d_inst_offsets.ptr, ctx->err))
    return B2E_ERR_NOMEM;
  return B2E_OK;
}

static int ensure_particle_buffers(b2e_ctx *ctx, int64_t n) {
  for (auto &c : ctx->d_cols)
    CUDA_TRY(ctx, c.ensure((size_t)n));
  CUDA_TRY(ctx, ctx->d_ids.ensure((size_t)n));
  CUDA_TRY(ctx, ctx->d_lost_pass.ensure((size_t)n));
  CUDA_TRY(ctx, ctx->d_lost_elem.ensure((size_t)n));
  CUDA_TRY(ctx, ctx->d_flag.ensure(1));
  CUDA_TRY(ctx, ctx->d_counters.ensure(2));
  return B2E_OK;
}

extern "C" int b2e_upload_particles(b2e_ctx *ctx, const double *const columns[6], const int64_t *ids, int64_t n) {
  if (!ctx || n < 0 || (n > 0 && (!columns || !ids)))
    return fail(ctx, B2E_ERR_ARG, "b2e_upload_particles: bad arguments");
  for (int c = 0; c < 6 && n > 0; c++)
    if (!columns[c])
      return fail(ctx, B2E_ERR_ARG, "b2e_upload_particles: column %d is null", c);
  cudaSetDevice(ctx->device);
  int rc = ensure_particle_buffers(ctx, n);
  if (rc)
    return rc;
  if (n > 0) {
    for (int c = 0; c < 6; c++)
      CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_cols[c].ptr, columns[c], sizeof(double) * n, cudaMemcpyHostToDevice,
                                    ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_ids.ptr, ids, sizeof(int64_t) * n, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_lost_pass.ptr, 0xff, sizeof(int32_t) * n, ctx->stream));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_lost_elem.ptr, 0xff, sizeof(int32_t) * n, ctx->stream));
  }
  ctx->n = n;
  ctx->particles_loaded = true;
  ctx->use_ext = false;
  ctx->pass_counter = 0;
  if (ctx->n_inst == 1) {
    ctx->inst_offsets = {0, n};
    build_tiles(ctx);
    return upload_lattice_tables(ctx);
  }
  if (ctx->inst_offsets.back() != n)
    return fail(ctx, B2E_ERR_ARG, "b2e_upload_particles: ensemble offsets cover %lld particles, got %lld",
                (long long)ctx->inst_offsets.back(), (long long)n);
  build_tiles(ctx); /* a compaction of the previous run may have shortened the tiles */
  return upload_tiles(ctx);
}

static DevParticles particle_view(b2e_ctx *ctx) {
  if (ctx->use_ext)
    return ctx->ext;
  DevParticles P;
  P.x = ctx->d_cols[0].ptr;
  P.xp = ctx->d_cols[1].ptr;
  P.y = ctx->d_cols[2].ptr;
  P.yp = ctx->d_cols[3].ptr;
  P.s = ctx->d_cols[4].ptr;
  P.dp = ctx->d_cols[5].ptr;
  P.lost_pass = ctx->d_lost_pass.ptr;
  P.lost_elem = ctx->d_lost_elem.ptr;
  return P;
}

/* Autotuner: time every ring-kernel variant on one pass of a scratch copy of
 * the current particle state (so the real state is untouched) and keep the
 * fastest.  The variants differ only in register allocation and in how often
 * a block's warps are brought back in step, never in arithmetic, so the
 * choice cannot change results.  With history recording the timed pass
 * records too (into slots the real launch overwrites). */
static int autotune_ring(b2e_ctx *ctx, const RingLaunch &Lreal, bool staged, size_t smem, int p, int e) {
  const int64_t n = ctx->n;
  const int ne = Lreal.n_elems;
  CUDA_TRY(ctx, ctx->d_scratch.ensure((size_t)n * 6));
  CUDA_TRY(ctx, ctx->d_scratch_loss.ensure((size_t)n * 2));
  RingLaunch L = Lreal;
  double *cols[6] = {Lreal.P.x, Lreal.P.xp, Lreal.P.y, Lreal.P.yp, Lreal.P.s, Lreal.P.dp};
  L.P.x = ctx->d_scratch.ptr;
  L.P.xp = L.P.x + n;
  L.P.y = L.P.xp + n;
  L.P.yp = L.P.y + n;
  L.P.s = L.P.yp + n;
  L.P.dp = L.P.s + n;
  L.P.lost_pass = ctx->d_scratch_loss.ptr;
  L.P.lost_elem = L.P.lost_pass + n;
  /* one full pass starting at (p, e) */
  L.pass_begin = p;
  L.elem_begin = e;
  L.pass_end = e == 0 ? p : p + 1;
  L.elem_end = e == 0 ? ne : e;
  cudaEvent_t ev0, ev1;
  CUDA_TRY(ctx, cudaEventCreate(&ev0));
  CUDA_TRY(ctx, cudaEventCreate(&ev1));
  double *dst[6] = {L.P.x, L.P.xp, L.P.y, L.P.yp, L.P.s, L.P.dp};
  float best = 1e30f;
  int best_v = 1;
  ctx->tune_ms.assign(B2E_RING_VARIANTS, 0.f);
  for (int v = 1; v <= B2E_RING_VARIANTS; v++) {
    for (int c = 0; c < 6; c++)
      CUDA_TRY(ctx, cudaMemcpyAsync(dst[c], cols[c], sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(L.P.lost_pass, Lreal.P.lost_pass, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaEventRecord(ev0, ctx->stream));
    CUDA_TRY(ctx, launch_ring(L, (int)ctx->tiles.size(), staged, staged ? smem : 0, ctx->stream, v));
    CUDA_TRY(ctx, cudaEventRecord(ev1, ctx->stream));
    CUDA_TRY(ctx, cudaEventSynchronize(ev1));
    float ms = 0;
    CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ev0, ev1));
    ctx->tune_ms[v - 1] = ms;
    if (ms < best) {
      best = ms;
      best_v = v;
    }
    ctx->launches++;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  ctx->tuned_variant = best_v;
  return B2E_OK;
}

/* Lost-particle compaction between launches: survivors of every instance to
 * the front of its range (rows reordered, IDs with them), tiles rebuilt over
 * the survivors only. */
static int compact_particles(b2e_ctx *ctx) {
  const size_t n = (size_t)ctx->n;
  for (auto &c : ctx->d_cmp_cols)
    CUDA_TRY(ctx, c.ensure(n));
  CUDA_TRY(ctx, ctx->d_cmp_ids.ensure(n));
  CUDA_TRY(ctx, ctx->d_cmp_lost_pass.ensure(n));
  CUDA_TRY(ctx, ctx->d_cmp_lost_elem.ensure(n));
  CUDA_TRY(ctx, ctx->d_alive_inst.ensure((size_t)ctx->n_inst));
  DevParticles dst;
  dst.x = ctx->d_cmp_cols[0].ptr;
  dst.xp = ctx->d_cmp_cols[1].ptr;
  dst.y = ctx->d_cmp_cols[2].ptr;
  dst.yp = ctx->d_cmp_cols[3].ptr;
  dst.s = ctx->d_cmp_cols[4].ptr;
  dst.dp = ctx->d_cmp_cols[5].ptr;
  dst.lost_pass = ctx->d_cmp_lost_pass.ptr;
  dst.lost_elem = ctx->d_cmp_lost_elem.ptr;
  CUDA_TRY(ctx, launch_compact(particle_view(ctx), ctx->d_ids.ptr, dst, ctx->d_cmp_ids.ptr, ctx->d_inst_offsets.ptr,
                               ctx->n_inst, ctx->d_alive_inst.ptr, ctx->stream));
  ctx->launches++;
  std::vector<int> alive(ctx->n_inst);
  CUDA_TRY(ctx, cudaMemcpyAsync(alive.data(), ctx->d_alive_inst.ptr, sizeof(int) * ctx->n_inst, cudaMemcpyDeviceToHost,
                                ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < 6; c++)
    std::swap(ctx->d_cols[c], ctx->d_cmp_cols[c]);
  std::swap(ctx->d_ids, ctx->d_cmp_ids);
  std::swap(ctx->d_lost_pass, ctx->d_cmp_lost_pass);
  std::swap(ctx->d_lost_elem, ctx->d_cmp_lost_elem);
  build_tiles(ctx, alive.data());
  return upload_tiles(ctx);
}

/* Track element range [(pb, eb), (pe, ee)) with ring launches, splitting at CSR elements. */
static int run_ring_range(b2e_ctx *ctx, int pb, int eb, int pe, int ee) {
  const int ne = (int)ctx->lat.elems.size();
  RingLaunch L;
  L.P = particle_view(ctx);
  L.tiles = ctx->d_tiles.ptr;
  L.elems = ctx->d_elems.ptr;
  L.aps = ctx->d_aps.ptr;
  L.rf = ctx->d_rf.ptr;
  L.n_elems = ne;
  L.n_aps = (int)ctx->lat.aps.size();
  L.n_rf = ctx->lat.n_rf;
  L.n_tiles = (int)ctx->tiles.size();
  L.g.p_central = ctx->opt.p_central;
  L.g.coord_limit = ctx->opt.coord_limit;
  L.g.slope_limit = ctx->opt.slope_limit;
  L.error_flag = ctx->d_flag.ptr;
  L.hist = ctx->opt.record_history && !ctx->use_ext ? ctx->d_hist_partials.ptr : nullptr;
  L.hist_pass0 = ctx->hist_pass0;
  L.hist_passes = ctx->hist_passes;
  L.rad = ctx->radiates;
  L.rads = ctx->d_rads.ptr;
  L.tbt = ctx->opt.record_tbt && !ctx->use_ext && ctx->tbt_records > 0 ? ctx->d_tbt.ptr : nullptr;
  L.tbt_pass0 = ctx->pass_counter;
  L.tbt_records = ctx->tbt_records;
  L.tbt_rows = ctx->n;
  L.ids = ctx->use_ext ? nullptr : ctx->d_ids.ptr;
  L.isr_seed = ctx->opt.isr_seed;
  L.sr_limit = ctx->opt.sr_gaussian_limit == 0 ? 3.0 : ctx->opt.sr_gaussian_limit;
  size_t smem = sizeof(DevElem) * ne + sizeof(DevAperture) * L.n_aps;
  bool staged = smem <= 200 * 1024;
  int ppl = ctx->opt.passes_per_launch > 0 ? ctx->opt.passes_per_launch : (1 << 30);
  const bool compact = ctx->opt.compact_every > 0 && !ctx->use_ext && !L.hist;
  if (compact)
    ppl = std::min(ppl, ctx->opt.compact_every);
  int variant = ctx->opt.ring_variant;
  if (variant < 1 || variant > B2E_RING_VARIANTS) {
    /* autotune once per context on a multi-pass range of a large enough beam */
    if (!ctx->tuned_variant && pe > pb && ctx->n >= 16384 && !L.rad) {
      int rc = autotune_ring(ctx, L, staged, smem, pb, eb);
      if (rc)
        return rc;
    }
    variant = ctx->tuned_variant ? ctx->tuned_variant : 1;
  }
  int p = pb, e = eb;
  while (p < pe || (p == pe && e < ee)) {
    /* end of this launch: at most ppl passes, never past (pe, ee) */
    int lp = p + ppl - 1 < pe ? p + ppl - 1 : pe;
    int le = lp == pe ? ee : ne;
    if (lp > p && le == 0) { /* (lp, 0) is the same point as (lp-1, ne) */
      lp -= 1;
      le = ne;
    }
    if (compact && e == 0 && p >= 1 && p > pb) {
      int rc = compact_particles(ctx);
      if (rc)
        return rc;
      L.P = particle_view(ctx);
      L.ids = ctx->d_ids.ptr; /* the IDs moved with the rows */
      L.tiles = ctx->d_tiles.ptr;
      L.n_tiles = (int)ctx->tiles.size();
    }
    L.pass_begin = p;
    L.elem_begin = e;
    L.pass_end = lp;
    L.elem_end = le;
    CUDA_TRY(ctx, launch_ring(L, (int)ctx->tiles.size(), staged, staged ? smem : 0, ctx->stream, variant));
    ctx->launches += ctx->tiles.empty() ? 0 : 1;
    if (le >= ne) {
      p = lp + 1;
      e = 0;
    } else {
      p = lp;
      e = le;
    }
  }
  return B2E_OK;
}

static int count_alive(b2e_ctx *ctx, int64_t *n_alive) {
  unsigned long long counters[2];
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
  CUDA_TRY(ctx, launch_effort(particle_view(ctx).lost_pass, ctx->n, 0, 0, ctx->d_counters.ptr,
                              ctx->d_counters.ptr + 1, ctx->stream));
  ctx->launches++;
  CUDA_TRY(ctx, cudaMemcpyAsync(counters, ctx->d_counters.ptr, sizeof(counters), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *n_alive = (int64_t)counters[1];
  return B2E_OK;
}

/* Record number of WATCH element ie on pass p in this call, -1 if it does not
 * record then (START_PASS, INTERVAL, END_PASS; sdds_support.c:738-741). */
static int watch_record_of(const b2e_ctx *ctx, int ie, int p) {
  const DevElem &d = ctx->lat.elems[ie];
  const int k = (int)d.c[WA_ORDINAL], step = (int)d.c[WA_INTERVAL], end = (int)d.c[WA_END];
  const int first = ctx->watch_first[k];
  if (first < 0 || p < first || (p - first) % step != 0 || (end >= 0 && p > end))
    return -1;
  return (int)(ctx->watch_rec0[k] + (p - first) / step);
}

static int track_impl(b2e_ctx *ctx, double *effort) {
  const int ne = (int)ctx->lat.elems.size();
  const int p0 = ctx->pass_counter;
  const int npass = p0 + ctx->opt.n_passes; /* one past the last pass of this call */
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_flag.ptr, 0, sizeof(unsigned int), ctx->stream));
  const bool record = ctx->opt.record_history && !ctx->use_ext && ctx->opt.n_passes > 0;
  if (p0 == 0)
    ctx->history.clear();
  ctx->tbt_records = 0;
  if (ctx->opt.record_tbt && !ctx->use_ext) {
    if (!ctx->lat.csr_elements.empty())
      return fail(ctx, B2E_ERR_LATTICE, "turn-by-turn recording is not available with CSR elements");
    if (ctx->opt.compact_every > 0)
      return fail(ctx, B2E_ERR_ARG, "turn-by-turn recording keeps rows in place: no compact_every");
    ctx->tbt_records = ctx->opt.n_passes + 1;
    ctx->tbt_rows = ctx->n;
    CUDA_TRY(ctx, ctx->d_tbt.ensure(std::max<size_t>((size_t)ctx->tbt_records * 4 * ctx->n, 1)));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_tbt.ptr, 0xff, sizeof(double) * (size_t)ctx->tbt_records * 4 * ctx->n,
                                  ctx->stream)); /* NaN until written */
    CUDA_TRY(ctx, launch_tbt_start(particle_view(ctx), ctx->n, ctx->d_tbt.ptr, ctx->stream));
  }
  /* WATCH records of this call: for each recording WATCH, its passes in
   * [p0, npass), record numbers in WATCH order then pass order */
  ctx->watch_rec_elem.clear();
  ctx->watch_rec_pass.clear();
  ctx->watch_on = false;
  if (ctx->watch_max_bytes > 0 && !ctx->lat.watch_elements.empty()) {
    const size_t nw = ctx->lat.watch_elements.size();
    std::vector<int64_t> &rec0 = ctx->watch_rec0;
    std::vector<int32_t> &first = ctx->watch_first;
    rec0.assign(nw, 0);
    first.assign(nw, -1);
    for (size_t k = 0; k < nw; k++) {
      const DevElem &d = ctx->lat.elems[ctx->lat.watch_elements[k]];
      const long start = (long)d.c[WA_START], end = (long)d.c[WA_END], step = (long)d.c[WA_INTERVAL];
      long f = start >= p0 ? start : start + ((p0 - start + step - 1) / step) * step;
      rec0[k] = (int64_t)ctx->watch_rec_pass.size();
      for (long q = f; q < npass && (end < 0 || q <= end); q += step) {
        if (first[k] < 0)
          first[k] = (int32_t)q;
        ctx->watch_rec_elem.push_back(ctx->lat.watch_elements[k]);
        ctx->watch_rec_pass.push_back((int32_t)q);
      }
    }
    const size_t records = ctx->watch_rec_pass.size();
    const double need = (double)records * 7 * (double)ctx->n * sizeof(double);
    if (need > (double)ctx->watch_max_bytes)
      return fail(ctx, B2E_ERR_ARG, "WATCH output of this call needs %.0f bytes of device memory; b2e_set_watch allows "
                  "%lld", need, (long long)ctx->watch_max_bytes);
    if (records > 0 && ctx->n > 0) {
      ctx->watch_rows = ctx->n;
      CUDA_TRY(ctx, ctx->d_watch.ensure(records * 7 * (size_t)ctx->n));
      CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_watch.ptr, 0xff, sizeof(double) * records * 7 * (size_t)ctx->n,
                                    ctx->stream)); /* NaN in the rows of lost particles */
      ctx->watch_on = true;
    }
  }
  if (record) {
    if (!ctx->lat.csr_elements.empty())
      return fail(ctx, B2E_ERR_LATTICE, "history recording is not available with CSR elements");
    ctx->hist_pass0 = p0;
    ctx->hist_passes = ctx->opt.n_passes;
    CUDA_TRY(ctx, ctx->d_hist_partials.ensure(std::max<size_t>(ctx->tiles.size(), 1) * ctx->hist_passes * 11));
    CUDA_TRY(ctx, ctx->d_hist_out.ensure((size_t)ctx->n_inst * ctx->hist_passes * 5));
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_hist_partials.ptr, 0,
                                  sizeof(double) * std::max<size_t>(ctx->tiles.size(), 1) * ctx->hist_passes * 11,
                                  ctx->stream));
  }
  if (p0 == 0) {
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_rf.ptr, 0, sizeof(DevRfState) * std::max(1, ctx->n_inst * ctx->lat.n_rf),
                                  ctx->stream));
    if (ctx->csr.enabled && ctx->csr.n_bunches != ctx->n_inst &&
        csr_set_bunches(ctx->csr, ctx->n_inst, ctx->d_inst_offsets.ptr, ctx->err))
      return B2E_ERR_NOMEM;
    csr_reset(ctx->csr);
    /* CHARGE (do_tracking.c:1324-1360): macro-particle charge = TOTAL / particles
     * at start; in an ensemble every instance is a bunch of charge TOTAL */
    std::vector<int64_t> sizes(ctx->csr.n_bunches);
    for (int b = 0; ctx->csr.enabled && b < ctx->csr.n_bunches; b++)
      sizes[b] = ctx->csr.n_bunches == 1 ? ctx->n : ctx->inst_offsets[b + 1] - ctx->inst_offsets[b];
    if (ctx->csr.enabled && csr_reduce_counts(ctx->csr, sizes, ctx->stream, ctx->err))
      return B2E_ERR_CUDA;
    for (int b = 0; ctx->csr.enabled && b < ctx->csr.n_bunches; b++) {
      const int64_t nb = sizes[b];
      double q = 0;
      for (const b2e_element &el : ctx->base)
        if (el.type == B2E_CHARGE) {
          if (nb)
            q = el.p[B2E_CHARGE_TOTAL] / nb;
          if (el.p[B2E_CHARGE_PER_PARTICLE])
            q = el.p[B2E_CHARGE_PER_PARTICLE];
        }
      ctx->csr.macro_charge[b] = q;
    }
  }
  /* stop points: every RFCA on pass 0 (fiducial), every CSR element on every
   * pass, every recording WATCH on the passes it records */
  int p = p0, e = 0, watched_e = -1, watched_p = -1;
  size_t next_rf = 0;
  while (p < npass) {
    int stop_e = ne, stop_kind = 0; /* 1 = RFCA fiducial, 2 = CSR element, 3 = WATCH record */
    for (int ie = e; ie < ne; ie++) {
      if (p == 0 && next_rf < ctx->lat.rf_elements.size() && ctx->lat.rf_elements[next_rf] == ie) {
        stop_e = ie;
        stop_kind = 1;
        break;
      }
      if (ctx->lat.elems[ie].kind == K_CSRCSBEND || ctx->lat.elems[ie].kind == K_CSRDRIFT) {
        stop_e = ie;
        stop_kind = 2;
        break;
      }
      if (ctx->watch_on && ctx->lat.elems[ie].kind == K_WATCH && !(ie == watched_e && p == watched_p) &&
          watch_record_of(ctx, ie, p) >= 0) {
        stop_e = ie;
        stop_kind = 3;
        break;
      }
    }
    if (stop_kind == 0) {
      /* nothing collective ahead on this pass; if the lattice has no CSR
       * elements (and no WATCH records), run all remaining passes in fused
       * launches */
      int last_pass = ctx->lat.csr_elements.empty() && !ctx->watch_on ? npass - 1 : p;
      int rc = run_ring_range(ctx, p, e, last_pass, ne);
      if (rc)
        return rc;
      p = last_pass + 1;
      e = 0;
      continue;
    }
    if (stop_e > e) {
      int rc = run_ring_range(ctx, p, e, p, stop_e);
      if (rc)
        return rc;
    }
    if (stop_kind == 3) {
      /* the particles alive at the WATCH on this pass (do_tracking.c:1626-1629) */
      const int r = watch_record_of(ctx, stop_e, p);
      CUDA_TRY(ctx, launch_watch_copy(particle_view(ctx), ctx->use_ext ? nullptr : ctx->d_ids.ptr, ctx->n,
                                      ctx->d_watch.ptr + (size_t)r * 7 * ctx->watch_rows, ctx->stream));
      ctx->launches++;
    } else if (stop_kind == 1) {
      ctx->launches++;
      CUDA_TRY(ctx, launch_fiducial(particle_view(ctx), ctx->d_inst_offsets.ptr, ctx->n_inst, ctx->d_elems.ptr, ne,
                                    stop_e, ctx->d_rf.ptr, ctx->lat.n_rf, ctx->opt.p_central,
                                    ctx->opt.fiducial_particles, ctx->d_flag.ptr, ctx->stream));
      next_rf++;
      /* the RFCA itself is tracked by the next ring launch */
      int rc = run_ring_range(ctx, p, stop_e, p, stop_e + 1);
      if (rc)
        return rc;
    } else {
      /* the collective step needs the number of particles alive at its entrance
       * (n_part > 1 decides whether CSR is computed at all, csbend.c:1987) */
      std::vector<int64_t> alive;
      ctx->csr.d_offsets = ctx->d_inst_offsets.ptr;
      int rc = csr_count_alive(ctx->csr, particle_view(ctx).lost_pass, ctx->n, alive, ctx->stream, ctx->err);
      if (rc)
        return rc;
      ctx->launches++;
      rc = csr_track_element(ctx->csr, ctx->d_elems.ptr, ctx->lat.elems[stop_e], particle_view(ctx), ctx->n, alive,
                             stop_e, p, ctx->stream, ctx->err, &ctx->launches);
      if (rc)
        return rc;
      const int iap = p == 0 ? ctx->lat.elems[stop_e].ap_pass0 : ctx->lat.elems[stop_e].ap_later;
      CUDA_TRY(ctx, launch_post_element_sweep(particle_view(ctx), ctx->n, iap >= 0 ? ctx->d_aps.ptr + iap : nullptr,
                                              p, stop_e, ctx->stream));
      ctx->launches++;
    }
    if (stop_kind == 3) {
      /* the WATCH element itself (a no-op, then the after-element checks)
       * goes with the next ring launch */
      watched_e = stop_e;
      watched_p = p;
      e = stop_e;
      continue;
    }
    e = stop_e + 1;
    if (e >= ne) {
      p++;
      e = 0;
    }
  }
  ctx->pass_counter = npass;
  if (record) {
    CUDA_TRY(ctx, launch_history_merge(ctx->d_hist_partials.ptr, ctx->hist_passes, ctx->d_tile_first.ptr,
                                       ctx->n_inst, ctx->d_hist_out.ptr, ctx->stream));
    ctx->launches++;
    std::vector<double> h((size_t)ctx->n_inst * ctx->hist_passes * 5);
    CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), ctx->d_hist_out.ptr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    /* [inst][pass][5] -> append as [pass][inst][5] */
    const size_t base = ctx->history.size();
    ctx->history.resize(base + h.size());
    for (int j = 0; j < ctx->hist_passes; j++)
      for (int i = 0; i < ctx->n_inst; i++)
        for (int k = 0; k < 5; k++)
          ctx->history[base + ((size_t)j * ctx->n_inst + i) * 5 + k] = h[((size_t)i * ctx->hist_passes + j) * 5 + k];
  }
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
  ctx->launches++;
  CUDA_TRY(ctx, launch_effort(particle_view(ctx).lost_pass, ctx->n, p0, npass, ctx->d_counters.ptr,
                              ctx->d_counters.ptr + 1, ctx->stream));
  unsigned long long counters[2];
  unsigned int flag = 0;
  CUDA_TRY(ctx, cudaMemcpyAsync(counters, ctx->d_counters.ptr, sizeof(counters), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaMemcpyAsync(&flag, ctx->d_flag.ptr, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (flag & 2u)
    return fail(ctx, B2E_ERR_DEVICE, "No available particle for RF cavity fiducialization (FIDUCIAL=pmaximum: "
                "no particle after the first has a higher momentum)");
  if (flag)
    return fail(ctx, B2E_ERR_DEVICE, "device reported error flag 0x%x (RFCA fiducial missing)", flag);
  if (effort)
    *effort = (double)counters[0];
  return B2E_OK;
}

extern "C" int b2e_track(b2e_ctx *ctx, double *effort) {
  if (!ctx)
    return B2E_ERR_ARG;
  if (!ctx->lattice_loaded || !ctx->particles_loaded)
    return fail(ctx, B2E_ERR_STATE, "b2e_track: load a lattice and particles first");
  cudaSetDevice(ctx->device);
  ctx->use_ext = false;
  return track_impl(ctx, effort);
}

extern "C" int b2e_download(b2e_ctx *ctx, double *const columns[6], int64_t *ids, int32_t *lost_pass,
                            int32_t *lost_element, int64_t *n_left) {
  if (!ctx)
    return B2E_ERR_ARG;
  if (!ctx->particles_loaded)
    return fail(ctx, B2E_ERR_STATE, "b2e_download: no particles");
  cudaSetDevice(ctx->device);
  const int64_t n = ctx->n;
  if (n > 0) {
    for (int c = 0; c < 6; c++)
      if (columns && columns[c])
        CUDA_TRY(ctx, cudaMemcpyAsync(columns[c], ctx->d_cols[c].ptr, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                      ctx->stream));
    if (ids)
      CUDA_TRY(ctx, cudaMemcpyAsync(ids, ctx->d_ids.ptr, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (lost_pass)
      CUDA_TRY(ctx, cudaMemcpyAsync(lost_pass, ctx->d_lost_pass.ptr, sizeof(int32_t) * n, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    if (lost_element)
      CUDA_TRY(ctx, cudaMemcpyAsync(lost_element, ctx->d_lost_elem.ptr, sizeof(int32_t) * n,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (n_left) {
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 2 * sizeof(unsigned long long), ctx->stream));
    ctx->launches++;
    CUDA_TRY(ctx, launch_effort(ctx->d_lost_pass.ptr, n, 0, 0, ctx->d_counters.ptr, ctx->d_counters.ptr + 1,
                                ctx->stream));
    unsigned long long counters[2];
    CUDA_TRY(ctx, cudaMemcpyAsync(counters, ctx->d_counters.ptr, sizeof(counters), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *n_left = (int64_t)counters[1];
  }
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return B2E_OK;
}

extern "C" int b2e_track_host(b2e_ctx *ctx, double *const columns[6], int64_t *ids, int64_t n, int32_t *lost_pass,
                              int32_t *lost_element, int64_t *n_left, double *effort) {
  int rc = b2e_upload_particles(ctx, (const double *const *)columns, ids, n);
  if (rc)
    return rc;
  rc = b2e_track(ctx, effort);
  if (rc)
    return rc;
  return b2e_download(ctx, columns, ids, lost_pass, lost_element, n_left);
}

extern "C" int b2e_track_device(b2e_ctx *ctx, double *const dev_columns[6], const int64_t *dev_ids, int64_t n,
                                int32_t *dev_lost_pass, int32_t *dev_lost_element, double *effort) {
  (void)dev_ids;
  if (!ctx || !dev_columns || !dev_lost_pass || !dev_lost_element || n < 0)
    return fail(ctx, B2E_ERR_ARG, "b2e_track_device: bad arguments");
  if (!ctx->lattice_loaded)
    return fail(ctx, B2E_ERR_STATE, "b2e_track_device: load a lattice first");
  cudaSetDevice(ctx->device);
  int rc = ensure_particle_buffers(ctx, 1);
  if (rc)
    return rc;
  if (ctx->n_inst == 1) {
    ctx->inst_offsets = {0, n};
    build_tiles(ctx);
    rc = upload_lattice_tables(ctx);
    if (rc)
      return rc;
  } else if (ctx->inst_offsets.back() != n)
    return fail(ctx, B2E_ERR_ARG, "b2e_track_device: ensemble offsets do not cover n particles");
  ctx->ext.x = dev_columns[0];
  ctx->ext.xp = dev_columns[1];
  ctx->ext.y = dev_columns[2];
  ctx->ext.yp = dev_columns[3];
  ctx->ext.s = dev_columns[4];
  ctx->ext.dp = dev_columns[5];
  ctx->ext.lost_pass = dev_lost_pass;
  ctx->ext.lost_elem = dev_lost_element;
  ctx->use_ext = true;
  ctx->n = n;
  ctx->pass_counter = 0; /* caller-owned buffers: every call is a new run */
  rc = track_impl(ctx, effort);
  ctx->use_ext = false;
  ctx->particles_loaded = false;
  return rc;
}

extern "C" int b2e_ensemble_history(b2e_ctx *ctx, int64_t *survivors, double *cx, double *cy, double *ex,
                                    double *ey) {
  if (!ctx)
    return B2E_ERR_ARG;
  if (!ctx->opt.record_history)
    return fail(ctx, B2E_ERR_STATE, "b2e_ensemble_history: run options did not request record_history");
  const size_t n_inst = (size_t)ctx->n_inst, n_pass = ctx->history.size() / (n_inst * 5);
  for (size_t i = 0; i < n_inst; i++)
    for (size_t j = 0; j < n_pass; j++) {
      const double *h = &ctx->history[(j * n_inst + i) * 5];
      const size_t o = i * n_pass + j;
      if (survivors)
        survivors[o] = (int64_t)h[0];
      if (cx)
        cx[o] = h[1];
      if (cy)
        cy[o] = h[2];
      if (ex)
        ex[o] = h[3];
      if (ey)
        ey[o] = h[4];
    }
  return B2E_OK;
}

extern "C" int64_t b2e_history_passes(const b2e_ctx *ctx) {
  return ctx && ctx->n_inst > 0 ? (int64_t)(ctx->history.size() / ((size_t)ctx->n_inst * 5)) : -1;
}

extern "C" int b2e_set_watch(b2e_ctx *ctx, int64_t max_bytes) {
  if (!ctx || max_bytes < 0)
    return B2E_ERR_ARG;
  ctx->watch_max_bytes = max_bytes;
  return B2E_OK;
}

extern "C" int b2e_watch_records(b2e_ctx *ctx, int32_t *n_records, int64_t *rows, int32_t *elements, int32_t *passes,
                                 int32_t capacity) {
  if (!ctx || !n_records || !rows)
    return B2E_ERR_ARG;
  const int32_t nr = ctx->watch_on ? (int32_t)ctx->watch_rec_pass.size() : 0;
  *n_records = nr;
  *rows = ctx->watch_on ? ctx->watch_rows : 0;
  for (int32_t r = 0; r < nr && r < capacity; r++) {
    if (elements)
      elements[r] = ctx->watch_rec_elem[r];
    if (passes)
      passes[r] = ctx->watch_rec_pass[r];
  }
  return B2E_OK;
}

extern "C" int b2e_watch_data(b2e_ctx *ctx, int32_t record, double *host_out) {
  if (!ctx || !host_out || !ctx->watch_on || record < 0 || record >= (int32_t)ctx->watch_rec_pass.size())
    return B2E_ERR_ARG;
  const size_t len = 7 * (size_t)ctx->watch_rows;
  CUDA_TRY(ctx, cudaMemcpyAsync(host_out, ctx->d_watch.ptr + (size_t)record * len, sizeof(double) * len,
                                cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return B2E_OK;
}

extern "C" int b2e_tbt(b2e_ctx *ctx, double *host_out, int64_t capacity, int64_t *written) {
  if (!ctx || !written || capacity < 0)
    return B2E_ERR_ARG;
  if (!ctx->opt.record_tbt || ctx->tbt_records <= 0)
    return fail(ctx, B2E_ERR_STATE, "b2e_tbt: no turn-by-turn data (set record_tbt and track)");
  const int64_t total = (int64_t)ctx->tbt_records * 4 * ctx->tbt_rows;
  *written = total;
  if (!host_out)
    return B2E_OK;
  if (capacity < total)
    return fail(ctx, B2E_ERR_ARG, "b2e_tbt: %lld values needed, capacity %lld", (long long)total,
                (long long)capacity);
  CUDA_TRY(ctx, cudaMemcpyAsync(host_out, ctx->d_tbt.ptr, sizeof(double) * total, cudaMemcpyDeviceToHost,
                                ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return B2E_OK;
}

extern "C" int b2e_tbt_tunes(b2e_ctx *ctx, int32_t first_record, int32_t n_records, double *nux, double *nuy,
                             double *ax, double *ay) {
  if (!ctx)
    return B2E_ERR_ARG;
  if (!ctx->opt.record_tbt || ctx->tbt_records <= 0)
    return fail(ctx, B2E_ERR_STATE, "b2e_tbt_tunes: no turn-by-turn data (set record_tbt and track)");
  if (first_record < 0 || n_records < 4 || n_records > 8192 || first_record + n_records > ctx->tbt_records)
    return fail(ctx, B2E_ERR_ARG, "b2e_tbt_tunes: window [%d, %d) outside 4..8192 records of the %d recorded",
                first_record, first_record + n_records, ctx->tbt_records);
  const int64_t rows = ctx->tbt_rows;
  if (rows == 0)
    return B2E_OK;
  cudaSetDevice(ctx->device);
  CUDA_TRY(ctx, ctx->d_naff.ensure((size_t)rows * 16));
  CUDA_TRY(ctx, ctx->d_naff_bad.ensure((size_t)rows));
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_naff_bad.ptr, 0, sizeof(int) * rows, ctx->stream));
  double *scratch = ctx->d_naff.ptr, *nu = ctx->d_naff.ptr + (size_t)rows * 12;
  CUDA_TRY(ctx, launch_tbt_tunes(ctx->d_tbt.ptr, rows, first_record, n_records, scratch, ctx->d_naff_bad.ptr, nu,
                                 ctx->stream));
  ctx->launches += 2;
  double *outs[4] = {nux, nuy, ax, ay};
  for (int k = 0; k < 4; k++)
    if (outs[k])
      CUDA_TRY(ctx, cudaMemcpyAsync(outs[k], nu + (size_t)k * rows, sizeof(double) * rows, cudaMemcpyDeviceToHost,
                                    ctx->stream));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return B2E_OK;
}

extern "C" int b2e_naff(const double *dev_signals, int64_t n_signals, int32_t n_points, double *dev_frequency,
                        double *dev_amplitude, double *dev_phase, void *stream) {
  if (n_signals < 0 || n_points < 4 || n_points > 8192 || (n_signals > 0 && (!dev_signals || !dev_frequency ||
                                                                             !dev_amplitude || !dev_phase)))
    return B2E_ERR_ARG;
  if (n_signals == 0)
    return B2E_OK;
  return launch_naff(dev_signals, n_signals, n_points, dev_frequency, dev_amplitude, dev_phase,
                     (cudaStream_t)stream) == cudaSuccess
             ? B2E_OK
             : B2E_ERR_CUDA;
}

extern "C" int b2e_csr_wakes(b2e_ctx *ctx, double *wakes, int64_t capacity, int64_t *written) {
  if (!ctx || !written)
    return B2E_ERR_ARG;
  return csr_copy_wakes(ctx->csr, wakes, capacity, written, ctx->err);
}

extern "C" int b2e_set_csr_pages(b2e_ctx *ctx, int32_t record) {
  if (!ctx)
    return B2E_ERR_ARG;
  ctx->csr.record_pages = record != 0;
  return B2E_OK;
}

extern "C" int b2e_set_csr_timing(b2e_ctx *ctx, int32_t on) {
  if (!ctx)
    return B2E_ERR_ARG;
  ctx->csr.time_wake = on != 0;
  return B2E_OK;
}

extern "C" int b2e_csr_timing(b2e_ctx *ctx, double *wake_ms, int64_t *kicks, int64_t *learned_kicks) {
  if (!ctx || !wake_ms || !kicks || !learned_kicks)
    return B2E_ERR_ARG;
  cudaSetDevice(ctx->device);
  return csr_wake_timing(ctx->csr, wake_ms, kicks, learned_kicks, ctx->err);
}

extern "C" int b2e_csr_pages(b2e_ctx *ctx, double *pages, int64_t capacity, int64_t *written) {
  if (!ctx || !written)
    return B2E_ERR_ARG;
  cudaSetDevice(ctx->device);
  return csr_copy_pages(ctx->csr, pages, capacity, written, ctx->err);
}

extern "C" int b2e_set_csr_surrogate(b2e_ctx *ctx, b2e_wakenet *net, const double feature_scales[3], double tolerance,
                                     int32_t gate_stride) {
  if (!ctx)
    return B2E_ERR_ARG;
  if (net && (!feature_scales || !(tolerance >= 0) || gate_stride < 1))
    return fail(ctx, B2E_ERR_ARG, "b2e_set_csr_surrogate: scales, a tolerance >= 0 and a stride >= 1 are required");
  if (net && wakenet_bins(net) < 128)
    return fail(ctx, B2E_ERR_ARG, "b2e_set_csr_surrogate: not a wake network");
  ctx->csr.net = net;
  if (net) {
    ctx->csr.sc_dens = (float)feature_scales[0];
    ctx->csr.sc_deriv = (float)feature_scales[1];
    ctx->csr.sc_target = (float)feature_scales[2];
    ctx->csr.gate_tol = tolerance;
    ctx->csr.gate_stride = gate_stride;
  }
  return B2E_OK;
}

extern "C" int b2e_csr_surrogate_stats(b2e_ctx *ctx, int64_t *evaluations, int64_t *fallbacks, double *gate_errors,
                                       int64_t capacity, int64_t *written) {
  if (!ctx)
    return B2E_ERR_ARG;
  unsigned long long c[2] = {0, 0};
  cudaSetDevice(ctx->device);
  if (ctx->csr.d_sur_counts)
    CUDA_TRY(ctx, cudaMemcpy(c, ctx->csr.d_sur_counts, sizeof(c), cudaMemcpyDeviceToHost));
  if (evaluations)
    *evaluations = (int64_t)c[0];
  if (fallbacks)
    *fallbacks = (int64_t)c[1];
  const int64_t n = std::min<int64_t>(capacity, ctx->csr.gate_values);
  if (gate_errors && n > 0)
    CUDA_TRY(ctx, cudaMemcpy(gate_errors, ctx->csr.d_gate_log, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (written)
    *written = gate_errors ? std::max<int64_t>(n, 0) : ctx->csr.gate_values;
  return B2E_OK;
}

extern "C" int b2e_set_csr_reducer(b2e_ctx *ctx, b2e_reduce_fn fn, void *user) {
  if (!ctx)
    return B2E_ERR_ARG;
  ctx->csr.reducer = fn;
  ctx->csr.reducer_user = fn ? user : nullptr;
  return B2E_OK;
}
