// capi.cu -- the C-ABI of libbem_b200.so: contexts, the native bem_* API and
// the drop-in seam with the reference's gfortran-mangled entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "bem_internal.h"

namespace bem {

int fail(bem_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return code;
}

void dev_free(bem_ctx* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

int cuda_fail(bem_ctx* ctx, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  return fail(ctx, e == cudaErrorMemoryAllocation ? BEM_ERR_NOMEM : BEM_ERR_CUDA, m);
}

// Reads the device status words after a synchronisation.
cudaError_t raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limit;
  int dev = 0;
  const cudaError_t de = cudaGetDevice(&dev);
  if (de != cudaSuccess) return de;
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = limit[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

int check_status(bem_ctx* ctx) {
  int st[ST_COUNT] = {0};
  BEM_CUDA(ctx, cudaMemcpyAsync(st, ctx->d_status, sizeof st, cudaMemcpyDeviceToHost, ctx->stream));
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (st[ST_TIMEOUT]) return fail(ctx, BEM_ERR_TIMEOUT, "a bounded device wait timed out");
  if (st[ST_SINGULAR]) return fail(ctx, BEM_ERR_SINGULAR, "zero pivot at column " + std::to_string(st[ST_SINGULAR]));
  if (st[ST_DEGENERATE]) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5");
  return BEM_OK;
}

static void free_mesh(bem_ctx* ctx, Mesh& m) {
  dev_free(ctx, m.gq);
  dev_free(ctx, m.eta);
  dev_free(ctx, m.colloc);
  dev_free(ctx, m.corner);
  dev_free(ctx, m.degen);
  m = Mesh{};
}

static void free_system(bem_ctx* ctx, System& s) {
  dev_free(ctx, s.A);
  dev_free(ctx, s.zh_pre);
  dev_free(ctx, s.zg_pre);
  dev_free(ctx, s.diag_h);
  dev_free(ctx, s.diag_g);
  dev_free(ctx, s.rhs_part);
  dev_free(ctx, s.x);
  s = System{};
}

static int ensure_system(bem_ctx* ctx, int nn, bool preswap) {
  System& s = ctx->sys;
  if (s.nn != nn || !s.A) {
    free_system(ctx, s);
    s.nn = nn;
    s.lda = (size_t)nn;
    BEM_CUDA(ctx, dev_alloc(ctx, &s.A, s.lda * (size_t)(nn + 1) * sizeof(double2)));
    const int nbe = (nn + 2) / 3;
    BEM_CUDA(ctx, dev_alloc(ctx, &s.diag_h, (size_t)nbe * 9 * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &s.diag_g, (size_t)nbe * 9 * sizeof(double2)));
  }
  if (preswap && !s.zh_pre) {
    BEM_CUDA(ctx, dev_alloc(ctx, &s.zh_pre, (size_t)nn * nn * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &s.zg_pre, (size_t)nn * nn * sizeof(double2)));
  }
  return BEM_OK;
}

static cudaEvent_t prof_event(bem_ctx* ctx) {
  Profiler& P = ctx->prof;
  if (P.used == P.pool.size()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    P.pool.push_back(e);
  }
  return P.pool[P.used++];
}

ProfScope::ProfScope(bem_ctx* c, int k, double work, double bytes) : ctx(c), cls(k) {
  Profiler& P = ctx->prof;
  if (!P.on) return;
  P.launches[k]++;
  P.work[k] += work;
  P.bytes[k] += bytes;
  cudaEvent_t a = prof_event(ctx);
  b = prof_event(ctx);
  cudaEventRecord(a, ctx->stream);
  P.recs.push_back(Profiler::Rec{k, a, b});
}

ProfScope::~ProfScope() {
  if (b) cudaEventRecord(b, ctx->stream);
}

}  // namespace bem

using namespace bem;

// ---------------------------------------------------------------------------
// Native API.
// ---------------------------------------------------------------------------
extern "C" {

const char* bem_status_string(int status) {
  switch (status) {
    case BEM_OK: return "ok";
    case BEM_ERR_DEGENERATE: return "degenerate Jacobian (DET < 1e-5)";
    case BEM_ERR_SINGULAR: return "singular matrix";
    case BEM_ERR_ARG: return "bad argument";
    case BEM_ERR_CUDA: return "CUDA error";
    case BEM_ERR_NOMEM: return "out of device memory";
    case BEM_ERR_STATE: return "call out of order";
    case BEM_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

const char* bem_last_error(bem_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

long long bem_ctx_launch_count(bem_ctx* ctx) { return ctx ? ctx->launches : 0; }

int bem_ctx_create(int device, bem_ctx** out) {
  if (!out) return BEM_ERR_ARG;
  *out = nullptr;
  bem_ctx* ctx = new bem_ctx();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  ctx->stream = ctx->own_stream;
  if (e == cudaSuccess) {
    // The device's stream-ordered pool keeps what contexts free, so that the
    // next context's buffers come from it without a new device allocation.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      unsigned long long keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    e = dev_alloc(ctx, &ctx->d_status, ST_WORDS * sizeof(int));
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status, 0, ST_WORDS * sizeof(int), ctx->stream);  // wait limit 0: the default
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return e == cudaErrorMemoryAllocation ? BEM_ERR_NOMEM : BEM_ERR_CUDA;
  }
  if (const char* env = getenv("BEM_TF32_MMA_SYNC")) ctx->use_tcgen05 = env[0] != '1';
  if (const char* env = getenv("BEM_TRSV_LEGACY")) ctx->use_trsv_coop = env[0] != '1';
  if (const char* env = getenv("BEM_LU_PAIRS")) ctx->lu_pairs = env[0] != '0';
  if (const char* env = getenv("BEM_GRAPHS")) ctx->use_graphs = env[0] != '0';
  if (const char* env = getenv("BEM_PANEL_CALU")) ctx->panel_calu = env[0] == '1';
  if (const char* env = getenv("BEM_PANEL_PUSH")) ctx->panel_push = env[0] != '0';
  if (const char* env = getenv("BEM_TRSV_INV")) ctx->trsv_inv = env[0] != '0';
  if (const char* env = getenv("BEM_LASWP_TC")) ctx->laswp_tc = env[0] != '0';
  if (const char* env = getenv("BEM_LU_QUADS")) ctx->lu_quads = env[0] != '0';
  if (const char* env = getenv("BEM_PANEL_ASYNC")) ctx->panel_async = env[0] != '0';
  if (const char* env = getenv("BEM_F64_PAIRS")) ctx->f64_pairs = env[0] != '0';
  if (const char* env = getenv("BEM_F64_CUBLAS")) ctx->f64_cublas = env[0] != '0';
  if (const char* env = getenv("BEM_TC_PAIR")) ctx->tc_pair = env[0] != '0';
  if (const char* env = getenv("BEM_SMALL_CLUSTERS")) ctx->small_clusters = env[0] != '0';
  if (const char* env = getenv("BEM_PANEL_TSLU")) ctx->panel_tslu = env[0] == '1';
  *out = ctx;
  return BEM_OK;
}

int bem_ctx_destroy(bem_ctx* ctx) {
  if (!ctx) return BEM_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  // everything of ctx is idle now: free it on the context's own stream (the
  // caller's stream may be gone by the time the frees run)
  ctx->stream = ctx->own_stream;
  free_mesh(ctx, ctx->mesh);
  free_system(ctx, ctx->sys);
  dev_free(ctx, ctx->hestdiag);
  dev_free(ctx, ctx->gestdiag);
  dev_free(ctx, ctx->zdfi);
  dev_free(ctx, ctx->kode);
  dev_free(ctx, ctx->d_status);
  dev_free(ctx, ctx->static_part);
  LuWork& L = ctx->lu;
  dev_free(ctx, L.ipiv);
  dev_free(ctx, L.perm);
  dev_free(ctx, L.slot_val);
  dev_free(ctx, L.slot_row);
  dev_free(ctx, L.cand);
  dev_free(ctx, L.drow);
  dev_free(ctx, L.barrier);
  dev_free(ctx, L.trsv_w);
  dev_free(ctx, L.tinv);
  dev_free(ctx, L.linv);
  dev_free(ctx, L.gmap);
  dev_free(ctx, L.trsv_ctr);
  dev_free(ctx, L.pstart);
  dev_free(ctx, L.ts_s);
  dev_free(ctx, L.ts_ipiv);
  dev_free(ctx, L.ts_perm);
  dev_free(ctx, L.ts_c);
  dev_free(ctx, L.ts_gid);
  dev_free(ctx, L.ts_cipiv);
  dev_free(ctx, L.ts_cperm);
  dev_free(ctx, L.lg);
  dev_free(ctx, ctx->grp_desc);
  for (bem_ctx* w : ctx->workers) bem_ctx_destroy(w);
  ctx->workers.clear();
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  release_sweep(ctx);
  release_interior(ctx);
  release_cublas(ctx);
  tc_release(ctx);
  for (cudaEvent_t e : ctx->prof.pool) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return BEM_OK;
}

int bem_ctx_set_stream(bem_ctx* ctx, void* stream) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  // work and frees already enqueued on the old stream finish before the
  // context's buffers are used, or freed, on the new one
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return BEM_OK;
}

int bem_sync(bem_ctx* ctx) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return check_status(ctx);
}

int bem_mesh_upload(bem_ctx* ctx, int n, int nbe, int np, int npg, const int* cone, const double* cx,
                    const double* cy, const double* cz, const double* cxm, const double* cym, const double* czm,
                    const double* etas, const double* gi, const double* ome) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (n <= 0 || nbe <= 0 || nbe > n || np <= 0 || npg <= 0 || npg > kMaxNpg || !cone || !cx || !cy || !cz ||
      !cxm || !cym || !czm || !etas || !gi || !ome)
    return fail(ctx, BEM_ERR_ARG, "bem_mesh_upload: bad sizes or null pointer");
  for (int i = 0; i < 4 * n; ++i)
    if (cone[i] < 1 || cone[i] > np) return fail(ctx, BEM_ERR_ARG, "bem_mesh_upload: node number out of range");
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  free_mesh(ctx, ctx->mesh);
  Mesh& m = ctx->mesh;
  m.n = n;
  m.nbe = nbe;
  m.np = np;
  m.npg = npg;
  m.ng = npg * npg;
  for (int i = 0; i < npg; ++i) {
    m.gi[i] = gi[i];
    m.ome[i] = ome[i];
  }
  BEM_CUDA(ctx, dev_alloc(ctx, &m.gq, (size_t)n * m.ng * sizeof(double4)));
  BEM_CUDA(ctx, dev_alloc(ctx, &m.eta, (size_t)n * sizeof(double4)));
  BEM_CUDA(ctx, dev_alloc(ctx, &m.colloc, (size_t)n * sizeof(double4)));
  BEM_CUDA(ctx, dev_alloc(ctx, &m.corner, (size_t)n * 12 * sizeof(double)));
  BEM_CUDA(ctx, dev_alloc(ctx, &m.degen, (size_t)n * sizeof(int)));
  // Staging copies of the raw mesh arrays (freed after the precompute).
  const size_t nd = (size_t)3 * np + 6 * (size_t)n;
  double* d_raw = nullptr;
  int* d_cone = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &d_raw, nd * sizeof(double)));
  BEM_CUDA(ctx, dev_alloc(ctx, &d_cone, (size_t)4 * n * sizeof(int)));
  double *dcx = d_raw, *dcy = dcx + np, *dcz = dcy + np, *detas = dcz + np, *dcxm = detas + 3 * (size_t)n,
         *dcym = dcxm + n, *dczm = dcym + n;
  cudaStream_t st = ctx->stream;
  BEM_CUDA(ctx, cudaMemcpyAsync(dcx, cx, np * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(dcy, cy, np * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(dcz, cz, np * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(detas, etas, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(dcxm, cxm, n * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(dcym, cym, n * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(dczm, czm, n * sizeof(double), cudaMemcpyHostToDevice, st));
  BEM_CUDA(ctx, cudaMemcpyAsync(d_cone, cone, 4 * (size_t)n * sizeof(int), cudaMemcpyHostToDevice, st));
  int rc = launch_geometry(ctx, dcx, dcy, dcz, d_cone, detas, dcxm, dcym, dczm);
  BEM_CUDA(ctx, cudaStreamSynchronize(st));
  dev_free(ctx, d_raw);
  dev_free(ctx, d_cone);
  if (rc) return rc;
  int flags[2];
  BEM_CUDA(ctx, cudaMemcpy(flags, ctx->d_status + ST_COUNT, sizeof flags, cudaMemcpyDeviceToHost));
  ctx->have_mesh = true;
  ctx->have_hest = ctx->have_gest = ctx->have_dyn = false;
  // Per-mesh buffers sized by nbe are reallocated on the next use.
  dev_free(ctx, ctx->zdfi);
  dev_free(ctx, ctx->kode);
  ctx->zdfi = nullptr;
  ctx->kode = nullptr;
  dev_free(ctx, ctx->static_part);
  ctx->static_part = nullptr;
  ctx->static_chunks = 0;
  release_sweep(ctx);
  ctx->sys.assembled = ctx->sys.solved = false;
  dev_free(ctx, ctx->hestdiag);
  dev_free(ctx, ctx->gestdiag);
  ctx->hestdiag = ctx->gestdiag = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &ctx->hestdiag, (size_t)nbe * 9 * sizeof(double)));
  BEM_CUDA(ctx, dev_alloc(ctx, &ctx->gestdiag, (size_t)nbe * 9 * sizeof(double)));
  // Remember the degenerate flags: [0] any element, [1] boundary elements.
  ctx->mesh_flag_all = flags[0];
  ctx->mesh_flag_bnd = flags[1];
  return BEM_OK;
}

int bem_ghmatece(bem_ctx* ctx, const double c[4], int compute_gest, double* hestdiag_out, double* gestdiag_out) {
  if (!ctx || !c) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "bem_ghmatece before bem_mesh_upload");
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  int rc = launch_static(ctx, c, compute_gest, nullptr);
  if (rc) return rc;
  const int nbe = ctx->mesh.nbe;
  if (hestdiag_out)
    BEM_CUDA(ctx, cudaMemcpyAsync(hestdiag_out, ctx->hestdiag, (size_t)nbe * 9 * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  if (gestdiag_out && compute_gest)
    BEM_CUDA(ctx, cudaMemcpyAsync(gestdiag_out, ctx->gestdiag, (size_t)nbe * 9 * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  rc = check_status(ctx);
  ctx->have_hest = true;
  if (compute_gest) ctx->have_gest = true;
  if (rc) return rc;
  if (ctx->mesh_flag_all) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on an element");
  return BEM_OK;
}

static int upload_diag(bem_ctx* ctx, double* dst, const double* src, bool& flag) {
  if (!ctx || !src) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "static diagonal before bem_mesh_upload");
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaMemcpyAsync(dst, src, (size_t)ctx->mesh.nbe * 9 * sizeof(double), cudaMemcpyHostToDevice,
                                ctx->stream));
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  flag = true;
  return BEM_OK;
}

int bem_set_gestdiag(bem_ctx* ctx, const double* g) { return upload_diag(ctx, ctx ? ctx->gestdiag : nullptr, g, ctx->have_gest); }
int bem_set_hestdiag(bem_ctx* ctx, const double* h) { return upload_diag(ctx, ctx ? ctx->hestdiag : nullptr, h, ctx->have_hest); }

int bem_static_h(bem_ctx* ctx, const double c[4], double* hest_out) {
  if (!ctx || !c || !hest_out) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "bem_static_h before bem_mesh_upload");
  cudaSetDevice(ctx->device);
  const size_t count = (size_t)3 * ctx->mesh.nbe * 3 * ctx->mesh.n;
  double* d = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &d, count * sizeof(double)));
  BEM_CUDA(ctx, cudaMemsetAsync(d, 0, count * sizeof(double), ctx->stream));
  int rc = launch_static(ctx, c, 0, d);
  if (!rc) {
    cudaError_t e = cudaMemcpyAsync(hest_out, d, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "copy static H");
  }
  if (!rc) rc = check_status(ctx);
  dev_free(ctx, d);
  if (!rc) ctx->have_hest = true;
  return rc;
}

int bem_dyn_upload(bem_ctx* ctx, const double* zdfi, const int* kode) {
  if (!ctx || !zdfi || !kode) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "bem_dyn_upload before bem_mesh_upload");
  cudaSetDevice(ctx->device);
  const int nn = 3 * ctx->mesh.nbe;
  if (!ctx->zdfi) {
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->zdfi, (size_t)nn * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->kode, (size_t)nn * sizeof(int)));
  }
  BEM_CUDA(ctx, cudaMemcpyAsync(ctx->zdfi, zdfi, (size_t)nn * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  BEM_CUDA(ctx, cudaMemcpyAsync(ctx->kode, kode, (size_t)nn * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  ctx->h_zdfi.assign(zdfi, zdfi + 2 * (size_t)nn);
  ctx->h_kode.assign(kode, kode + nn);
  ctx->have_dyn = true;
  return BEM_OK;
}

int bem_ghmatecd(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                 double fr, int flags) {
  if (!ctx || !zge || !zcs || !zcp || !c) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh || !ctx->have_dyn) return fail(ctx, BEM_ERR_STATE, "bem_ghmatecd needs mesh and BCs");
  if ((flags & BEM_FAST_SINGULAR) && (!ctx->have_hest || !ctx->have_gest))
    return fail(ctx, BEM_ERR_STATE, "bem_ghmatecd needs HESTdiag and GESTdiag");
  if (ctx->mesh.ng * (int)sizeof(double4) > 1024 * 32)
    return fail(ctx, BEM_ERR_ARG, "Gauss rule too large");
  cudaSetDevice(ctx->device);
  int rc = ensure_system(ctx, 3 * ctx->mesh.nbe, (flags & BEM_KEEP_PRESWAP) != 0);
  if (rc) return rc;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  rc = launch_dynamic(ctx, zge, zcs, zcp, c, fr, flags);
  if (rc) return rc;
  ctx->sys.assembled = true;
  ctx->sys.solved = false;
  ctx->sys.have_preswap = (flags & BEM_KEEP_PRESWAP) != 0;
  ctx->assembled_mesh = true;
  ctx->sys.zge_last = make_double2(zge[0], zge[1]);
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  return BEM_OK;
}

int bem_get_system(bem_ctx* ctx, double* zh, double* zfi) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->sys.assembled || ctx->sys.solved) return fail(ctx, BEM_ERR_STATE, "no assembled system");
  cudaSetDevice(ctx->device);
  const System& s = ctx->sys;
  if (zh)
    BEM_CUDA(ctx, cudaMemcpy2DAsync(zh, (size_t)s.nn * sizeof(double2), s.A, s.lda * sizeof(double2),
                                    (size_t)s.nn * sizeof(double2), s.nn, cudaMemcpyDeviceToHost, ctx->stream));
  if (zfi)
    BEM_CUDA(ctx, cudaMemcpyAsync(zfi, s.A + (size_t)s.nn * s.lda, (size_t)s.nn * sizeof(double2),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  return check_status(ctx);
}

int bem_get_preswap(bem_ctx* ctx, double* zh, double* zg) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->sys.have_preswap) return fail(ctx, BEM_ERR_STATE, "assemble with BEM_KEEP_PRESWAP first");
  cudaSetDevice(ctx->device);
  const size_t bytes = (size_t)ctx->sys.nn * ctx->sys.nn * sizeof(double2);
  if (zh) BEM_CUDA(ctx, cudaMemcpyAsync(zh, ctx->sys.zh_pre, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  if (zg) BEM_CUDA(ctx, cudaMemcpyAsync(zg, ctx->sys.zg_pre, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  return check_status(ctx);
}

int bem_linsolve(bem_ctx* ctx, double* zfi_out) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->sys.assembled || ctx->sys.solved) return fail(ctx, BEM_ERR_STATE, "bem_linsolve without an assembled system");
  cudaSetDevice(ctx->device);
  int rc = lu_factor_solve(ctx);
  if (rc) return rc;
  ctx->sys.solved = true;
  const System& s = ctx->sys;
  if (zfi_out)
    BEM_CUDA(ctx, cudaMemcpyAsync(zfi_out, s.A + (size_t)s.nn * s.lda, (size_t)s.nn * sizeof(double2),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  return check_status(ctx);
}

int bem_solve_dense(bem_ctx* ctx, int nn, const double* a, const double* b, double* x) {
  if (!ctx || nn <= 0 || !a || !b || !x) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  int rc = ensure_system(ctx, nn, false);
  if (rc) return rc;
  System& s = ctx->sys;
  BEM_CUDA(ctx, cudaMemcpy2DAsync(s.A, s.lda * sizeof(double2), a, (size_t)nn * sizeof(double2),
                                  (size_t)nn * sizeof(double2), nn, cudaMemcpyHostToDevice, ctx->stream));
  BEM_CUDA(ctx, cudaMemcpyAsync(s.A + (size_t)nn * s.lda, b, (size_t)nn * sizeof(double2), cudaMemcpyHostToDevice,
                                ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  s.assembled = true;
  s.solved = false;
  s.have_preswap = false;
  rc = lu_factor_solve(ctx);
  if (rc) return rc;
  s.solved = true;
  BEM_CUDA(ctx, cudaMemcpyAsync(x, s.A + (size_t)nn * s.lda, (size_t)nn * sizeof(double2), cudaMemcpyDeviceToHost,
                                ctx->stream));
  return check_status(ctx);
}

int bem_static_solve(bem_ctx* ctx, const double c[4], double ge, const int* kode, const double* dfi, double* disp,
                     double* trac) {
  if (!ctx || !c || !kode || !dfi || !disp || !trac) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh || !ctx->have_hest || !ctx->have_gest)
    return fail(ctx, BEM_ERR_STATE, "bem_static_solve needs the mesh, HESTdiag and GESTdiag");
  cudaSetDevice(ctx->device);
  const int nn = 3 * ctx->mesh.nbe;
  int rc = ensure_system(ctx, nn, false);
  if (rc) return rc;
  System& s = ctx->sys;
  double* Gs = nullptr;
  double* d_dfi = nullptr;
  int* d_kode = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &Gs, (size_t)nn * nn * sizeof(double)));
  BEM_CUDA(ctx, dev_alloc(ctx, &d_dfi, (size_t)nn * sizeof(double)));
  BEM_CUDA(ctx, dev_alloc(ctx, &d_kode, (size_t)nn * sizeof(int)));
  BEM_CUDA(ctx, cudaMemcpyAsync(d_dfi, dfi, (size_t)nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  BEM_CUDA(ctx, cudaMemcpyAsync(d_kode, kode, (size_t)nn * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  rc = launch_static_system(ctx, c, ge, d_kode, d_dfi, s.A, s.lda, Gs);
  s.assembled = true;
  s.solved = false;
  s.have_preswap = false;
  if (!rc) rc = lu_factor_solve(ctx);
  std::vector<double2> x((size_t)nn);
  if (!rc) {
    s.solved = true;
    BEM_CUDA(ctx, cudaMemcpyAsync(x.data(), s.A + (size_t)nn * s.lda, (size_t)nn * sizeof(double2),
                                  cudaMemcpyDeviceToHost, ctx->stream));
    rc = check_status(ctx);
  }
  cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, Gs);
  dev_free(ctx, d_dfi);
  dev_free(ctx, d_kode);
  if (rc) return rc;
  // Interec.for:59-67 with the real GE.
  for (int i = 0; i < nn; ++i) {
    if (kode[i] == 0) {
      disp[i] = dfi[i];
      trac[i] = x[i].x * ge;
    } else {
      disp[i] = x[i].x;
      trac[i] = dfi[i];
    }
  }
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  return BEM_OK;
}

int bem_linsolve_async(bem_ctx* ctx) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->sys.assembled || ctx->sys.solved) return fail(ctx, BEM_ERR_STATE, "bem_linsolve without an assembled system");
  cudaSetDevice(ctx->device);
  int rc = lu_factor_solve(ctx);
  if (rc) return rc;
  ctx->sys.solved = true;
  return BEM_OK;
}

int bem_sweep(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
              const double* freqs, int nfreq, int form, int batch, int refine, double* x_out, double* corr_out) {
  if (!ctx || !zge || !zcs || !zcp || !c || (nfreq > 0 && !freqs)) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh || !ctx->have_dyn || !ctx->have_hest || !ctx->have_gest)
    return fail(ctx, BEM_ERR_STATE, "bem_sweep needs the mesh, BCs and static diagonals");
  cudaSetDevice(ctx->device);
  int rc = sweep(ctx, zge, zcs, zcp, c, freqs, nfreq, form, batch, refine, x_out, corr_out);
  if (rc) return rc;
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  return BEM_OK;
}

int bem_sweep_async(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                    const double* freqs, int nfreq, int form, int batch, int refine, double* x_out) {
  if (!ctx || !zge || !zcs || !zcp || !c || (nfreq > 0 && !freqs)) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh || !ctx->have_dyn || !ctx->have_hest || !ctx->have_gest)
    return fail(ctx, BEM_ERR_STATE, "bem_sweep_async needs the mesh, BCs and static diagonals");
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  cudaSetDevice(ctx->device);
  return sweep(ctx, zge, zcs, zcp, c, freqs, nfreq, form, batch, refine, x_out, nullptr, false);
}

int bem_batch_solve(bem_ctx* driver, int nprob, bem_ctx* const* probs, const double* freqs, const double* zge,
                    const double* zcs, const double* zcp, const double* c, int form, int refine,
                    double* const* x_out, double* corr_out) {
  if (!driver || nprob < 0 || (nprob > 0 && (!probs || !freqs || !zge || !zcs || !zcp || !c))) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(driver->mu);
  for (int p = 0; p < nprob; ++p) {
    bem_ctx* pc = probs[p];
    if (!pc || pc == driver) return fail(driver, BEM_ERR_ARG, "bem_batch_solve: bad problem context");
    if (pc->device != driver->device) return fail(driver, BEM_ERR_ARG, "bem_batch_solve: contexts on other devices");
    if (!pc->have_mesh || !pc->have_dyn || !pc->have_hest || !pc->have_gest)
      return fail(driver, BEM_ERR_STATE, "bem_batch_solve: a problem lacks mesh, BCs or static diagonals");
    if (pc->mesh.ng * (int)sizeof(double4) > 1024 * 32) return fail(driver, BEM_ERR_ARG, "Gauss rule too large");
  }
  cudaSetDevice(driver->device);
  return batch_solve(driver, nprob, probs, freqs, zge, zcs, zcp, c, form, refine, x_out, corr_out);
}

static bool* option_slot(bem_ctx* ctx, const char* name) {
  if (!strcmp(name, "tcgen05")) return &ctx->use_tcgen05;
  if (!strcmp(name, "trsv_coop")) return &ctx->use_trsv_coop;
  if (!strcmp(name, "trsv_inv")) return &ctx->trsv_inv;
  if (!strcmp(name, "laswp_tc")) return &ctx->laswp_tc;
  if (!strcmp(name, "lu_pairs")) return &ctx->lu_pairs;
  if (!strcmp(name, "lu_quads")) return &ctx->lu_quads;
  if (!strcmp(name, "f64_pairs")) return &ctx->f64_pairs;
  if (!strcmp(name, "f64_cublas")) return &ctx->f64_cublas;
  if (!strcmp(name, "tc_pair")) return &ctx->tc_pair;
  if (!strcmp(name, "small_clusters")) return &ctx->small_clusters;
  if (!strcmp(name, "panel_tslu")) return &ctx->panel_tslu;
  if (!strcmp(name, "panel_calu")) return &ctx->panel_calu;
  if (!strcmp(name, "panel_push")) return &ctx->panel_push;
  if (!strcmp(name, "panel_async")) return &ctx->panel_async;
  if (!strcmp(name, "graphs")) return &ctx->use_graphs;
  return nullptr;
}

// Integer options: CTA budgets for a context that shares its GPU with
// another one running at the same time (0 = the whole device).
static int* int_option_slot(bem_ctx* ctx, const char* name) {
  if (!strcmp(name, "gemm_ctas")) return &ctx->gemm_ctas;
  if (!strcmp(name, "trsv_ctas")) return &ctx->trsv_ctas;
  return nullptr;
}

constexpr int kWaitLimitMaxMs = 60000;

int bem_ctx_set_option(bem_ctx* ctx, const char* name, int value) {
  if (!ctx || !name) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!strcmp(name, "wait_limit_ms")) {
    // kept in the context's device status words: every bounded wait reads it
    // at the start of its kernel, captured graphs included
    if (value < 1 || value > kWaitLimitMaxMs)
      return fail(ctx, BEM_ERR_ARG, "wait_limit_ms must be in 1..60000");
    const unsigned long long ns = (unsigned long long)value * 1000000ull;
    cudaSetDevice(ctx->device);
    BEM_CUDA(ctx, cudaMemcpyAsync(ctx->d_status + ST_WAIT_LIMIT, &ns, sizeof ns, cudaMemcpyHostToDevice,
                                  ctx->stream));
    BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->wait_limit_ms = value;
    return BEM_OK;
  }
  bool* slot = option_slot(ctx, name);
  int* islot = slot ? nullptr : int_option_slot(ctx, name);
  if (!slot && !islot) return fail(ctx, BEM_ERR_ARG, std::string("unknown option ") + name);
  if (islot && value < 0) return fail(ctx, BEM_ERR_ARG, std::string("negative value for ") + name);
  const bool changed = slot ? *slot != (value != 0) : *islot != value;
  if (changed) {
    if (slot) *slot = value != 0;
    else *islot = value;
    cudaSetDevice(ctx->device);
    release_sweep_graph(ctx);  // a captured step may embody the old choice
  }
  return BEM_OK;
}

int bem_ctx_get_option(bem_ctx* ctx, const char* name, int* value) {
  if (!ctx || !name || !value) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!strcmp(name, "wait_limit_ms")) {
    *value = ctx->wait_limit_ms;
    return BEM_OK;
  }
  if (bool* slot = option_slot(ctx, name)) {
    *value = *slot ? 1 : 0;
    return BEM_OK;
  }
  if (int* islot = int_option_slot(ctx, name)) {
    *value = *islot;
    return BEM_OK;
  }
  return fail(ctx, BEM_ERR_ARG, std::string("unknown option ") + name);
}

int bem_sweep_batch_limit(bem_ctx* ctx, int form, int* limit) {
  if (!ctx || !limit || (form != BEM_FORM_PLAIN && form != BEM_FORM_MIXED)) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "bem_sweep_batch_limit needs the mesh");
  cudaSetDevice(ctx->device);
  *limit = lu_lockstep_capacity(ctx, 3 * ctx->mesh.nbe, form == BEM_FORM_MIXED);
  return BEM_OK;
}

int bem_prof_enable(bem_ctx* ctx, int on) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->prof.on = on != 0;
  return BEM_OK;
}

int bem_prof_reset(bem_ctx* ctx) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  Profiler& P = ctx->prof;
  P.recs.clear();
  P.used = 0;
  for (int c = 0; c < BEM_PROF_CLASSES; ++c) {
    P.ms[c] = 0.0;
    P.launches[c] = 0;
    P.work[c] = 0.0;
    P.bytes[c] = 0.0;
  }
  return BEM_OK;
}

int bem_prof_bytes(bem_ctx* ctx, double* bytes) {
  if (!ctx || !bytes) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (int c = 0; c < BEM_PROF_CLASSES; ++c) bytes[c] = ctx->prof.bytes[c];
  return BEM_OK;
}

int bem_prof_read(bem_ctx* ctx, double* ms, long long* launches, double* work) {
  if (!ctx) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  Profiler& P = ctx->prof;
  for (const auto& r : P.recs) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) P.ms[r.cls] += t;
  }
  P.recs.clear();
  P.used = 0;
  for (int c = 0; c < BEM_PROF_CLASSES; ++c) {
    if (ms) ms[c] = P.ms[c];
    if (launches) launches[c] = P.launches[c];
    if (work) work[c] = P.work[c];
  }
  return BEM_OK;
}

int bem_wait_selftest(bem_ctx* ctx, int which) {
  if (!ctx || (which != 0 && which != 1)) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return wait_selftest(ctx, which);
}

int bem_measure_fp64_peak(bem_ctx* ctx, double* tflops) {
  if (!ctx || !tflops) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  return measure_fp64_peak(ctx, tflops);
}

int bem_interior(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], double rho, double fr,
                 int l, const double* cxi, const double* cyi, const double* czi, const double* disp,
                 const double* trac, double* zdsol, double* zssol) {
  if (!ctx || !zge || !zcs || !zcp || l < 0 || (l > 0 && (!cxi || !cyi || !czi || !disp || !trac || !zdsol)))
    return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->have_mesh) return fail(ctx, BEM_ERR_STATE, "bem_interior needs the mesh");
  if (ctx->mesh.ng * (int)sizeof(double4) > 1024 * 32) return fail(ctx, BEM_ERR_ARG, "Gauss rule too large");
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  int rc = interior_points(ctx, zge, zcs, zcp, rho, fr, l, cxi, cyi, czi, disp, trac, zdsol, zssol);
  if (rc) return rc;
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  return BEM_OK;
}

int bem_measure_peaks(bem_ctx* ctx, double* out) {
  if (!ctx || !out) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  int rc = measure_fma_peaks(ctx, &out[0], &out[1]);
  if (!rc) rc = measure_fp64_peak(ctx, &out[2]);
  if (!rc) rc = measure_tf32_peak(ctx, 128, &out[3]);
  if (!rc) rc = measure_tf32_peak(ctx, 256, &out[4]);
  return rc;
}

int bem_unswap(bem_ctx* ctx, double* disp_out, double* trac_out) {
  if (!ctx || !disp_out || !trac_out) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->sys.solved || !ctx->have_dyn || (int)ctx->h_kode.size() != ctx->sys.nn)
    return fail(ctx, BEM_ERR_STATE, "bem_unswap before bem_linsolve");
  cudaSetDevice(ctx->device);
  const System& s = ctx->sys;
  const int nn = s.nn;
  BEM_CUDA(ctx, cudaMemcpyAsync(disp_out, s.A + (size_t)nn * s.lda, (size_t)nn * sizeof(double2),
                                cudaMemcpyDeviceToHost, ctx->stream));
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // Interec.for:59-67: for KODE=0, ZCH = ZFI*ZGE; ZFI = ZDFI; ZDFI = ZCH.
  const double gr = s.zge_last.x, gi = s.zge_last.y;
  for (int i = 0; i < nn; ++i) {
    double zr = ctx->h_zdfi[2 * i], zi = ctx->h_zdfi[2 * i + 1];
    if (ctx->h_kode[i] == 0) {
      double xr = disp_out[2 * i], xi = disp_out[2 * i + 1];
      trac_out[2 * i] = xr * gr - xi * gi;
      trac_out[2 * i + 1] = xr * gi + xi * gr;
      disp_out[2 * i] = zr;
      disp_out[2 * i + 1] = zi;
    } else {
      trac_out[2 * i] = zr;
      trac_out[2 * i + 1] = zi;
    }
  }
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// Drop-in seam: one process-wide context, as the reference's device globals.
// ---------------------------------------------------------------------------
static bem_ctx* g_ctx = nullptr;
static std::mutex g_mu;

static bem_ctx* seam_ctx() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ctx) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (bem_ctx_create(dev, &g_ctx) != BEM_OK) {
      fputs("libbem_b200: could not create the CUDA context\n", stderr);
      exit(1);
    }
  }
  return g_ctx;
}

// CUDA and solver failures end the program, as cuda_assert (src/kernels/shared.cu:33-41).
static void seam_check(int rc, const char* where) {
  if (rc == BEM_OK || rc == BEM_ERR_DEGENERATE) return;
  fprintf(stderr, "%s: %s (%s)\n", where, bem_status_string(rc), bem_last_error(g_ctx));
  exit(1);
}

void send_shared_data_to_gpu_(double cx[], double cy[], double cz[], double cxm[], double cym[], double czm[],
                              double etas[], double gi[], double ome[], int cone[], int* np, int* npg, int* n,
                              int* nbe) {
  bem_ctx* ctx = seam_ctx();
  seam_check(bem_mesh_upload(ctx, *n, *nbe, *np, *npg, cone, cx, cy, cz, cxm, cym, czm, etas, gi, ome),
             "send_shared_data_to_gpu");
}

void send_dyn_data_gpu_(int* nbe, double zdfi[], int kode[]) {
  bem_ctx* ctx = seam_ctx();
  (void)nbe;
  seam_check(bem_dyn_upload(ctx, zdfi, kode), "send_dyn_data_gpu");
}

void cuda_ghmatece_(int* nbe, int* npg, int* n, int* np, double* c3, double* c4, double* fr, double hestdiag[],
                    int* status) {
  (void)nbe; (void)npg; (void)n; (void)np; (void)fr; (void)hestdiag;
  bem_ctx* ctx = seam_ctx();
  const double c[4] = {0.0, 0.0, *c3, *c4};
  int rc = bem_ghmatece(ctx, c, 0, nullptr, nullptr);
  seam_check(rc, "cuda_ghmatece");
  *status = (rc == BEM_ERR_DEGENERATE) ? 1 : 0;
}

void cuda_send_gest_data_(int* nbe, double* gestdiag) {
  (void)nbe;
  bem_ctx* ctx = seam_ctx();
  seam_check(bem_set_gestdiag(ctx, gestdiag), "cuda_send_gest_data");
}

void cuda_ghmatecd_(int* nbe, int* npg, int* n, int* np, double zge[2], double zcs[2], double zcp[2], double* c1,
                    double* c2, double* c3, double* c4, double* fr, double hestdiag[], double gestdiag[],
                    double zfi[], double zhp[], int kode[], int* fast_singular, int* status) {
  (void)nbe; (void)npg; (void)n; (void)np; (void)hestdiag; (void)gestdiag; (void)zfi; (void)zhp; (void)kode;
  bem_ctx* ctx = seam_ctx();
  const double c[4] = {*c1, *c2, *c3, *c4};
  int rc = bem_ghmatecd(ctx, zge, zcs, zcp, c, *fr, *fast_singular ? BEM_FAST_SINGULAR : 0);
  seam_check(rc, "cuda_ghmatecd");
  *status = (rc == BEM_ERR_DEGENERATE) ? 1 : 0;
}

void cuda_linsolve_(int* nn, int* n, double zh[], double zfi[]) {
  (void)nn; (void)n; (void)zh;
  bem_ctx* ctx = seam_ctx();
  int rc = bem_linsolve(ctx, zfi);
  if (rc == BEM_ERR_SINGULAR) {
    fputs("ERRO: Matriz ZH singular\n", stderr);  // lu_assert, src/kernels/Linsolve_cu.cu:10-17
    exit(1);
  }
  seam_check(rc, "cuda_linsolve");
}

void cuda_interec1_(int* n, int* nbe, int* npg, int* l, int* np, double cxi[], double cyi[], double czi[],
                    double zge[2], double zcs[2], double zcp[2], double* c1, double* c2, double* c3, double* c4,
                    double* fr, double zdfi[], double zfi[], double zdsol[], int* status) {
  (void)n; (void)nbe; (void)npg; (void)np; (void)c1; (void)c2; (void)c3; (void)c4;
  bem_ctx* ctx = seam_ctx();
  int rc = bem_interior(ctx, zge, zcs, zcp, 0.0, *fr, *l, cxi, cyi, czi, zfi, zdfi, zdsol, nullptr);
  seam_check(rc, "cuda_interec1");
  *status = (rc == BEM_ERR_DEGENERATE) ? 1 : 0;
}

void deallocate_shared_gpu_data_(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  bem_ctx_destroy(g_ctx);
  g_ctx = nullptr;
}

}  // extern "C"
