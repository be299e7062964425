// mixed.cu -- the batching and precision forms of the frequency sweep.
//
// bem_sweep assembles and solves a list of frequencies on the resident mesh,
// `batch` problems at a time in lockstep (one launch per kernel for the whole
// batch: assembly, every LU step, every refinement step).
//
//   plain form:  FP64 assembly, FP64 LU (as bem_ghmatecd + bem_linsolve).
//   mixed form:  FP64 assembly that also stores a complex64 copy of the
//                system; LU of the copy in FP32 with TF32 tensor-core trailing
//                updates; then iterative refinement in FP64:
//                  x <- x0;  repeat: r = b - A x (FP64, the FP64 matrix),
//                                    d = LU32^-1 r (FP32 factors),
//                                    x <- x + d (FP64).
//                The relative size of the last correction, max|d| / max|x|,
//                is reported per frequency.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "bem_internal.h"

namespace bem {

namespace {

constexpr int kResidRows = 256, kResidCols = 256;

// partial[prob][chunk][r] = sum over the chunk's columns c of A(r,c) x(c).
__global__ void __launch_bounds__(kResidRows) k_resid_partial(const double2* __restrict__ A, size_t lda,
                                                              size_t a_stride, const double2* __restrict__ x,
                                                              size_t x_stride, int nn, int chunks, double2* part) {
  __shared__ double2 s_x[kResidCols];
  const int prob = blockIdx.z;
  const double2* Ap = A + (size_t)prob * a_stride;
  const double2* xp = x + (size_t)prob * x_stride;
  const int c0 = blockIdx.y * kResidCols;
  const int cn = min(kResidCols, nn - c0);
  for (int i = threadIdx.x; i < cn; i += blockDim.x) s_x[i] = xp[c0 + i];
  __syncthreads();
  const int r = blockIdx.x * kResidRows + threadIdx.x;
  if (r >= nn) return;
  double re = 0.0, im = 0.0;
  for (int c = 0; c < cn; ++c) {
    const double2 a = Ap[(size_t)(c0 + c) * lda + r];
    const double2 xv = s_x[c];
    re = fma(a.x, xv.x, fma(-a.y, xv.y, re));
    im = fma(a.x, xv.y, fma(a.y, xv.x, im));
  }
  part[((size_t)prob * chunks + blockIdx.y) * nn + r] = make_double2(re, im);
}

// v32 = (complex64)(b - sum of partials), b = column nn of A.
__global__ void k_resid_final(const double2* __restrict__ A, size_t lda, size_t a_stride,
                              const double2* __restrict__ part, int nn, int chunks, float2* v, size_t v_stride) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  const int prob = blockIdx.y;
  const double2 b = A[(size_t)prob * a_stride + (size_t)nn * lda + r];
  double re = b.x, im = b.y;
  const double2* pp = part + (size_t)prob * chunks * nn;
  for (int c = 0; c < chunks; ++c) {
    const double2 q = pp[(size_t)c * nn + r];
    re -= q.x;
    im -= q.y;
  }
  v[(size_t)prob * v_stride + r] = make_float2((float)re, (float)im);
}

// x = (complex128) column nn of the FP32 system (the first, FP32, solution).
// y = sum of the partials (y = A x), FP64.
__global__ void k_gemv_final(const double2* __restrict__ part, int nn, int chunks, double2* y) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  double re = 0.0, im = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const double2 q = part[(size_t)c * nn + r];
    re += q.x;
    im += q.y;
  }
  y[r] = make_double2(re, im);
}

__global__ void k_x_init(const float2* __restrict__ A32, size_t lda, size_t a_stride, int nn, double2* x,
                         size_t x_stride) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  const int prob = blockIdx.y;
  const float2 v = A32[(size_t)prob * a_stride + (size_t)nn * lda + r];
  x[(size_t)prob * x_stride + r] = make_double2(v.x, v.y);
}

// x += d; tracks max|d| and max|x| (|re|+|im|) per problem in norm[prob][2].
__global__ void k_ir_update(double2* x, size_t x_stride, const float2* __restrict__ d, size_t d_stride, int nn,
                            unsigned long long* norm) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int prob = blockIdx.y;
  double dm = 0.0, xm = 0.0;
  if (r < nn) {
    const float2 dv = d[(size_t)prob * d_stride + r];
    double2 xv = x[(size_t)prob * x_stride + r];
    xv.x += dv.x;
    xv.y += dv.y;
    x[(size_t)prob * x_stride + r] = xv;
    dm = fabs((double)dv.x) + fabs((double)dv.y);
    xm = fabs(xv.x) + fabs(xv.y);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, off));
    xm = fmax(xm, __shfl_xor_sync(0xffffffffu, xm, off));
  }
  if ((threadIdx.x & 31) == 0) {
    // Non-negative doubles order like their bit patterns.
    atomicMax(&norm[2 * prob], __double_as_longlong(dm));
    atomicMax(&norm[2 * prob + 1], __double_as_longlong(xm));
  }
}


void free_sweep(bem_ctx* ctx, SweepBuf& S) {
  dev_free(ctx, S.A64);
  dev_free(ctx, S.A32);
  dev_free(ctx, S.x64);
  dev_free(ctx, S.v32);
  dev_free(ctx, S.part);
  dev_free(ctx, S.diag_h);
  dev_free(ctx, S.diag_g);
  dev_free(ctx, S.rhs_part);
  dev_free(ctx, S.norm);
  dev_free(ctx, S.G64);
  S = SweepBuf{};
}

int ensure_sweep(bem_ctx* ctx, int batch, bool mixed, bool keep_g = false) {
  SweepBuf& S = ctx->sweep;
  const int nn = 3 * ctx->mesh.nbe;
  const int nbe = ctx->mesh.nbe;
  const int chunks = rhs_chunks(ctx);
  if (S.nn == nn && S.batch >= batch && (!mixed || S.A32) && (!keep_g || S.G64) && S.rhs_chunks >= chunks)
    return BEM_OK;
  // A captured step names these buffers: let it finish and drop it before they go.
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  release_sweep_graph(ctx);
  free_sweep(ctx, S);
  S.nn = nn;
  S.batch = batch;
  S.lda = (size_t)((nn + 1) & ~1);  // even: 16-byte aligned column strides for the FP32 TMA maps
  S.a_stride = S.lda * (size_t)(nn + 1);
  S.rhs_chunks = chunks;
  S.resid_chunks = (nn + kResidCols - 1) / kResidCols;
  BEM_CUDA(ctx, dev_alloc(ctx, &S.A64, S.a_stride * batch * sizeof(double2)));
  if (mixed) BEM_CUDA(ctx, dev_alloc(ctx, &S.A32, S.a_stride * batch * sizeof(float2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.x64, (size_t)nn * batch * sizeof(double2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.v32, (size_t)nn * batch * sizeof(float2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.part, (size_t)S.resid_chunks * nn * batch * sizeof(double2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.diag_h, (size_t)nbe * 9 * batch * sizeof(double2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.diag_g, (size_t)nbe * 9 * batch * sizeof(double2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.rhs_part, (size_t)chunks * nn * batch * sizeof(double2)));
  BEM_CUDA(ctx, dev_alloc(ctx, &S.norm, (size_t)2 * batch * (kMaxRefine + 1) * sizeof(unsigned long long)));
  if (keep_g) BEM_CUDA(ctx, dev_alloc(ctx, &S.G64, S.a_stride * batch * sizeof(double2)));
  return BEM_OK;
}

// `iters` refinement steps on the first `bsz` problems of S, the k-th step's
// norms in slot it0 + k: r = b - A64 x (FP64, b = column nn), d = LU32^-1 r,
// x += d.
int refine_steps(bem_ctx* ctx, SweepBuf& S, int bsz, int iters, int it0) {
  const int nn = S.nn;
  const dim3 vgrid((nn + 255) / 256, bsz);
  for (int it = 0; it < iters; ++it) {
    {
      ProfScope ps(ctx, 5, 8.0 * (double)nn * nn * bsz, 16.0 * (double)nn * nn * bsz);
      k_resid_partial<<<dim3((nn + kResidRows - 1) / kResidRows, S.resid_chunks, bsz), kResidRows, 0,
                        ctx->stream>>>(S.A64, S.lda, S.a_stride, S.x64, nn, nn, S.resid_chunks, S.part);
      k_resid_final<<<vgrid, 256, 0, ctx->stream>>>(S.A64, S.lda, S.a_stride, S.part, nn, S.resid_chunks, S.v32,
                                                    nn);
    }
    ctx->launches += 2;
    int rc = lu_solve_vec(ctx, S.A32, S.lda, S.a_stride, nn, bsz, S.v32, nn, true);
    if (rc) return rc;
    k_ir_update<<<vgrid, 256, 0, ctx->stream>>>(S.x64, nn, S.v32, nn, nn, S.norm + (size_t)2 * bsz * (it0 + it));
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
  }
  return BEM_OK;
}

}  // namespace

static void drop_sweep_graph(bem_ctx* ctx) {
  if (ctx->sweep_exec) cudaGraphExecDestroy(ctx->sweep_exec);
  if (ctx->sweep_graph) cudaGraphDestroy(ctx->sweep_graph);
  ctx->sweep_exec = nullptr;
  ctx->sweep_graph = nullptr;
  ctx->sweep_dyn_nodes.clear();
}

void release_sweep_graph(bem_ctx* ctx) {
  drop_sweep_graph(ctx);
  ctx->sw_nn = 0;
}

void release_sweep(bem_ctx* ctx) {
  drop_sweep_graph(ctx);
  ctx->sw_nn = 0;
  free_sweep(ctx, ctx->sweep);
  free_sweep(ctx, ctx->bbuf);
}

int sweep(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
          const double* freqs, int nfreq, int form, int batch, int iters, double* x_out, double* corr_out,
          bool wait_out) {
  const bool mixed = form == BEM_FORM_MIXED;
  if (!mixed && form != BEM_FORM_PLAIN) return fail(ctx, BEM_ERR_ARG, "unknown form");
  if (batch < 1 || batch > kMaxBatch || nfreq < 0 || iters < 0 || iters > kMaxRefine)
    return fail(ctx, BEM_ERR_ARG, "bem_sweep: batch, count or refinement steps out of range");
  // No more problems in lockstep than the panel kernel keeps resident at once.
  batch = std::min(batch, lu_lockstep_capacity(ctx, 3 * ctx->mesh.nbe, mixed));
  int rc = ensure_sweep(ctx, batch, mixed);
  if (rc) return rc;
  SweepBuf& S = ctx->sweep;
  const int nn = S.nn;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  std::vector<unsigned long long> hnorm;
  // One lockstep step: assembly, LU (+ refinement) of `bsz` problems.
  auto enqueue = [&](const DynBatch& db, int bsz) -> int {
    int r = launch_dynamic_batch(ctx, db);
    if (r) return r;
    const dim3 vgrid((nn + 255) / 256, bsz);
    if (mixed) {
      r = lu_factor_solve_batch(ctx, S.A32, S.lda, S.a_stride, nn, bsz, true);
      if (r) return r;
      k_x_init<<<vgrid, 256, 0, ctx->stream>>>(S.A32, S.lda, S.a_stride, nn, S.x64, nn);
      ctx->launches++;
      BEM_CUDA(ctx, cudaMemsetAsync(S.norm, 0, (size_t)2 * bsz * kMaxRefine * sizeof(unsigned long long),
                                    ctx->stream));
      return refine_steps(ctx, S, bsz, iters, 0);
    }
    return lu_factor_solve_batch(ctx, S.A64, S.lda, S.a_stride, nn, bsz, false);
  };
  for (int f0 = 0; f0 < nfreq; f0 += batch) {
    const int bsz = std::min(batch, nfreq - f0);
    DynBatch db{};
    db.zge = zge;
    db.zcs = zcs;
    db.zcp = zcp;
    db.c = c;
    db.freqs = freqs + f0;
    db.batch = bsz;
    db.flags = BEM_FAST_SINGULAR;
    db.A = S.A64;
    db.lda = S.lda;
    db.a_stride = S.a_stride;
    db.A32 = mixed ? S.A32 : nullptr;
    db.diag_h = S.diag_h;
    db.diag_g = S.diag_g;
    db.rhs_part = S.rhs_part;
    // Steps after the first (which allocates and warms everything) run as one
    // CUDA graph: captured once per (size, batch, form), then replayed with
    // the new frequencies written into its assembly nodes.
    const bool warm = ctx->sw_nn == nn && ctx->sw_bsz == bsz && ctx->sw_mixed == (int)mixed &&
                      ctx->sw_iters == iters;  // a step of this shape already ran directly
    const bool graph = ctx->use_graphs && !ctx->prof.on && warm && bsz == batch;
    const bool have = ctx->sweep_exec && ctx->sg_nn == nn && ctx->sg_bsz == bsz &&
                      ctx->sg_mixed == (int)mixed && ctx->sg_iters == iters &&
                      ctx->sg_epoch == ctx->alloc_epoch;  // none of its buffers moved since
    if (graph && have) {
      rc = dyn_graph_update(ctx, ctx->sweep_exec, ctx->sweep_dyn_nodes, db);
      if (rc) return rc;
      BEM_CUDA(ctx, cudaGraphLaunch(ctx->sweep_exec, ctx->stream));
      ctx->launches += ctx->sg_launches;
    } else if (graph) {
      drop_sweep_graph(ctx);
      const long long l0 = ctx->launches;
      BEM_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const int erc = enqueue(db, bsz);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
      cudaGraphExec_t ex = nullptr;
      bool ok = erc == BEM_OK && ce == cudaSuccess && g &&
                cudaGraphInstantiate(&ex, g, 0) == cudaSuccess &&
                dyn_graph_nodes(ctx, g, ctx->sweep_dyn_nodes) == BEM_OK;
      cudaGetLastError();
      if (ok) {
        ctx->sweep_graph = g;
        ctx->sweep_exec = ex;
        ctx->sg_nn = nn;
        ctx->sg_bsz = bsz;
        ctx->sg_mixed = (int)mixed;
        ctx->sg_iters = iters;
        ctx->sg_epoch = ctx->alloc_epoch;
        ctx->sg_launches = ctx->launches - l0;
        BEM_CUDA(ctx, cudaGraphLaunch(ex, ctx->stream));
      } else {
        // The stream cannot be captured here: run the step directly from now on.
        if (ex) cudaGraphExecDestroy(ex);
        if (g) cudaGraphDestroy(g);
        ctx->sweep_dyn_nodes.clear();
        ctx->use_graphs = false;
        ctx->launches = l0;
        rc = enqueue(db, bsz);
        if (rc) return rc;
      }
    } else {
      rc = enqueue(db, bsz);
      if (rc) return rc;
      ctx->sw_nn = nn;
      ctx->sw_bsz = bsz;
      ctx->sw_mixed = (int)mixed;
      ctx->sw_iters = iters;
    }
    if (x_out) {
      double* dst = x_out + (size_t)2 * nn * f0;
      if (mixed)
        BEM_CUDA(ctx, cudaMemcpyAsync(dst, S.x64, (size_t)nn * bsz * sizeof(double2), cudaMemcpyDeviceToHost,
                                      ctx->stream));
      else
        BEM_CUDA(ctx, cudaMemcpy2DAsync(dst, (size_t)nn * sizeof(double2), S.A64 + (size_t)nn * S.lda,
                                        S.a_stride * sizeof(double2), (size_t)nn * sizeof(double2), bsz,
                                        cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (corr_out) {
      if (mixed && iters > 0) {
        hnorm.assign((size_t)2 * bsz * kMaxRefine, 0ull);
        BEM_CUDA(ctx, cudaMemcpyAsync(hnorm.data(), S.norm, (size_t)2 * bsz * iters * sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, ctx->stream));
        BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        const size_t last = (size_t)2 * bsz * (iters - 1);
        for (int b = 0; b < bsz; ++b) {
          double dm, xm;
          const unsigned long long du = hnorm[last + 2 * b], xu = hnorm[last + 2 * b + 1];
          memcpy(&dm, &du, sizeof dm);
          memcpy(&xm, &xu, sizeof xm);
          corr_out[f0 + b] = xm > 0 ? dm / xm : 0.0;
        }
      } else {
        for (int b = 0; b < bsz; ++b) corr_out[f0 + b] = 0.0;
      }
    }
  }
  if ((x_out && wait_out) || corr_out) return check_status(ctx);
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// Problems of uneven size (bem_batch_solve): sorted by size and grouped into
// classes whose largest member is at most 1.25 x the smallest and whose count
// fits the lockstep limit; each class is embedded in one padded size (the
// problem, then the identity) and runs through the lockstep LU of bem_sweep.
// A class is assembled in three launches (launch_dynamic_group: every member
// from its own context's mesh, static diagonals and BCs, straight into its
// padded slot) and its solutions come back in one copy, so the host issues a
// few dozen calls per class, not per problem.
// ---------------------------------------------------------------------------
namespace {

struct BatchNeed {
  size_t a_elems = 0, vec_elems = 0, resid_elems = 0, rhs_elems = 0, diag_elems = 0;
  int norm_batch = 0;
  void add(int npad, int batch, size_t diag, size_t rhs) {
    const size_t lda = (size_t)((npad + 1) & ~1), a_stride = lda * (size_t)(npad + 1);
    a_elems = std::max(a_elems, a_stride * batch);
    vec_elems = std::max(vec_elems, (size_t)npad * batch);
    resid_elems = std::max(resid_elems, (size_t)((npad + kResidCols - 1) / kResidCols) * npad * batch);
    rhs_elems = std::max(rhs_elems, rhs);
    diag_elems = std::max(diag_elems, diag);
    norm_batch = std::max(norm_batch, batch);
  }
};

// Sizes a worker's padded-system buffers for every class it will run.
int ensure_batchbuf(bem_ctx* d, const BatchNeed& q, bool mixed) {
  SweepBuf& S = d->bbuf;
  const bool fits = S.A64 && q.a_elems <= S.a_stride && (!mixed || S.A32) && q.vec_elems <= (size_t)S.nn &&
                    q.resid_elems <= (size_t)S.resid_chunks && q.rhs_elems <= (size_t)S.rhs_chunks &&
                    q.diag_elems <= (size_t)S.batch && (size_t)q.norm_batch <= S.norm_cap;
  if (fits) return BEM_OK;
  free_sweep(d, S);
  BEM_CUDA(d, dev_alloc(d, &S.A64, q.a_elems * sizeof(double2)));
  if (mixed) BEM_CUDA(d, dev_alloc(d, &S.A32, q.a_elems * sizeof(float2)));
  BEM_CUDA(d, dev_alloc(d, &S.x64, q.vec_elems * sizeof(double2)));
  BEM_CUDA(d, dev_alloc(d, &S.v32, q.vec_elems * sizeof(float2)));
  BEM_CUDA(d, dev_alloc(d, &S.part, q.resid_elems * sizeof(double2)));
  BEM_CUDA(d, dev_alloc(d, &S.diag_h, q.diag_elems * sizeof(double2)));
  BEM_CUDA(d, dev_alloc(d, &S.diag_g, q.diag_elems * sizeof(double2)));
  BEM_CUDA(d, dev_alloc(d, &S.rhs_part, q.rhs_elems * sizeof(double2)));
  BEM_CUDA(d, dev_alloc(d, &S.norm, (size_t)2 * q.norm_batch * (kMaxRefine + 1) * sizeof(unsigned long long)));
  // capacities, in elements (this buffer set is only read through views)
  S.a_stride = q.a_elems;
  S.nn = (int)q.vec_elems;
  S.resid_chunks = (int)q.resid_elems;
  S.rhs_chunks = (int)q.rhs_elems;
  S.batch = (int)q.diag_elems;
  S.norm_cap = (size_t)q.norm_batch;
  return BEM_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

constexpr int kBatchWorkers = 8;

int batch_solve(bem_ctx* d, int nprob, bem_ctx* const* probs, const double* freqs, const double* zge,
                const double* zcs, const double* zcp, const double* c, int form, int iters, double* const* x_out,
                double* corr_out) {
  const bool mixed = form == BEM_FORM_MIXED;
  if (!mixed && form != BEM_FORM_PLAIN) return fail(d, BEM_ERR_ARG, "unknown form");
  if (iters < 0 || iters > kMaxRefine) return fail(d, BEM_ERR_ARG, "refinement steps out of range");
  std::vector<int> order(nprob);
  for (int i = 0; i < nprob; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) { return probs[a]->mesh.nbe < probs[b]->mesh.nbe; });
  // Worker contexts: classes go round-robin to their streams and run concurrently.
  while ((int)d->workers.size() < kBatchWorkers) {
    bem_ctx* w = nullptr;
    const int rc = bem_ctx_create(d->device, &w);
    if (rc) return fail(d, rc, "bem_batch_solve: worker context");
    d->workers.push_back(w);
  }
  // Plan: size classes in sorted order, round-robin over the workers, each
  // worker's buffers sized once for all its classes (no allocation between
  // launches).
  struct Cls {
    int g0, g1, npad;
    size_t sol;  // offset of its solutions in the pinned staging, in double2
  };
  std::vector<Cls> plan;
  std::vector<BatchNeed> need_w(kBatchWorkers);
  size_t sol_total = 0;
  for (int g0 = 0; g0 < nprob;) {
    const int n0 = 3 * probs[order[g0]]->mesh.nbe;
    int g1 = g0 + 1, npad = n0;
    while (g1 < nprob) {
      const int n1 = 3 * probs[order[g1]]->mesh.nbe;
      if (n1 * 4 > n0 * 5) break;
      if (g1 - g0 + 1 > std::min(kMaxBatch, lu_lockstep_capacity(d, n1, mixed))) break;
      npad = n1;
      ++g1;
    }
    size_t diag = 0, rhs = 0;
    for (int k = g0; k < g1; ++k) {
      diag += (size_t)9 * probs[order[k]]->mesh.nbe;
      rhs += (size_t)rhs_chunks(probs[order[k]]) * 3 * probs[order[k]]->mesh.nbe;
    }
    need_w[plan.size() % kBatchWorkers].add(npad, g1 - g0, diag, rhs);
    plan.push_back({g0, g1, npad, sol_total});
    sol_total += (size_t)(g1 - g0) * npad;
    g0 = g1;
  }
  for (int w = 0; w < kBatchWorkers; ++w) {
    if (need_w[w].a_elems == 0) continue;
    const int rc = ensure_batchbuf(d->workers[w], need_w[w], mixed);
    if (rc) return fail(d, rc, std::string("bem_batch_solve: ") + d->workers[w]->last_error);
  }
  // Pinned staging: assembly descriptors, solutions, refinement norms.
  const size_t desc_bytes = dyn_problem_bytes();
  const size_t desc_total = align256((size_t)nprob * desc_bytes);
  const size_t norm_words = (size_t)nprob * 2 * (kMaxRefine + 1);
  const size_t need = desc_total + align256(sol_total * sizeof(double2)) + norm_words * sizeof(unsigned long long);
  if (d->pinned_bytes < need) {
    if (d->pinned) cudaFreeHost(d->pinned);
    d->pinned = nullptr;
    d->pinned_bytes = 0;
    BEM_CUDA(d, cudaMallocHost(&d->pinned, need));
    d->pinned_bytes = need;
  }
  if (d->grp_desc_bytes < desc_total) {
    dev_free(d, d->grp_desc);
    d->grp_desc = nullptr;
    d->grp_desc_bytes = 0;
    BEM_CUDA(d, dev_alloc(d, &d->grp_desc, desc_total));
    BEM_CUDA(d, cudaStreamSynchronize(d->stream));  // the workers' streams use it next
    d->grp_desc_bytes = desc_total;
  }
  unsigned char* hdesc = static_cast<unsigned char*>(d->pinned);
  unsigned char* ddesc = static_cast<unsigned char*>(d->grp_desc);
  double2* hsol = reinterpret_cast<double2*>(hdesc + desc_total);
  unsigned long long* hnorm = reinterpret_cast<unsigned long long*>(
      reinterpret_cast<unsigned char*>(hsol) + align256(sol_total * sizeof(double2)));
  std::vector<int> class_of(nprob), slot_of(nprob);
  for (bem_ctx* w : d->workers) BEM_CUDA(w, cudaMemsetAsync(w->d_status, 0, ST_COUNT * sizeof(int), w->stream));
  std::vector<GroupMember> mem;
  for (int ncls = 0; ncls < (int)plan.size(); ++ncls) {
    bem_ctx* wk = d->workers[ncls % kBatchWorkers];
    const int g0 = plan[ncls].g0, g1 = plan[ncls].g1, npad = plan[ncls].npad;
    const int B = g1 - g0;
    int rc = BEM_OK;
    SweepBuf& S = wk->bbuf;
    const size_t lda = (size_t)((npad + 1) & ~1), a_stride = lda * (size_t)(npad + 1);
    mem.assign(B, GroupMember{});
    size_t diag_off = 0, rhs_off = 0;
    for (int k = g0; k < g1; ++k) {
      const int p = order[k], slot = k - g0;
      class_of[p] = ncls;
      slot_of[p] = slot;
      bem_ctx* pc = probs[p];
      GroupMember& g = mem[slot];
      g.pc = pc;
      g.zge = zge + 2 * p;
      g.zcs = zcs + 2 * p;
      g.zcp = zcp + 2 * p;
      g.c = c + 4 * p;
      g.fr = freqs[p];
      g.A = S.A64 + (size_t)slot * a_stride;
      g.A32 = mixed ? S.A32 + (size_t)slot * a_stride : nullptr;
      g.lda = lda;
      g.npad = npad;
      g.diag_h = S.diag_h + diag_off;
      g.diag_g = S.diag_g + diag_off;
      g.rhs_part = S.rhs_part + rhs_off;
      diag_off += (size_t)9 * pc->mesh.nbe;
      rhs_off += (size_t)rhs_chunks(pc) * 3 * pc->mesh.nbe;
    }
    {
      const long long l0 = wk->launches;
      rc = launch_dynamic_group(wk, mem.data(), B, hdesc + (size_t)g0 * desc_bytes, ddesc + (size_t)g0 * desc_bytes);
      d->launches += wk->launches - l0;
      if (rc) return fail(d, rc, std::string("assembly of a batched class: ") + wk->last_error);
    }
    // the padded class through the lockstep LU (+ refinement)
    SweepBuf V = S;  // a view with this class's size for refine_steps
    V.nn = npad;
    V.lda = lda;
    V.a_stride = a_stride;
    V.resid_chunks = (npad + kResidCols - 1) / kResidCols;
    const long long l0 = wk->launches;
    if (mixed) {
      rc = lu_factor_solve_batch(wk, V.A32, lda, a_stride, npad, B, true);
      if (!rc) {
        k_x_init<<<dim3((npad + 255) / 256, B), 256, 0, wk->stream>>>(V.A32, lda, a_stride, npad, V.x64, npad);
        wk->launches++;
        rc = cudaMemsetAsync(V.norm, 0, (size_t)2 * B * (kMaxRefine + 1) * sizeof(unsigned long long),
                             wk->stream) == cudaSuccess
                 ? refine_steps(wk, V, B, iters, 0)
                 : BEM_ERR_CUDA;
      }
    } else {
      rc = lu_factor_solve_batch(wk, V.A64, lda, a_stride, npad, B, false);
    }
    d->launches += wk->launches - l0;
    if (rc) return fail(d, rc, std::string("bem_batch_solve: ") + wk->last_error);
    // the class's solutions (npad each, padding included) in one copy
    double2* dst = hsol + plan[ncls].sol;
    if (mixed)
      BEM_CUDA(d, cudaMemcpyAsync(dst, V.x64, (size_t)B * npad * sizeof(double2), cudaMemcpyDeviceToHost,
                                  wk->stream));
    else
      BEM_CUDA(d, cudaMemcpy2DAsync(dst, (size_t)npad * sizeof(double2), V.A64 + (size_t)npad * lda,
                                    a_stride * sizeof(double2), (size_t)npad * sizeof(double2), B,
                                    cudaMemcpyDeviceToHost, wk->stream));
    if (mixed && iters > 0)
      BEM_CUDA(d, cudaMemcpyAsync(hnorm + (size_t)2 * (kMaxRefine + 1) * g0, V.norm,
                                  (size_t)2 * B * (kMaxRefine + 1) * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, wk->stream));
  }
  for (bem_ctx* w : d->workers) {
    BEM_CUDA(d, cudaStreamSynchronize(w->stream));
    const int rc = check_status(w);
    if (rc) return fail(d, rc, std::string("bem_batch_solve: ") + w->last_error);
  }
  for (int p = 0; p < nprob; ++p) {
    if (probs[p]->mesh_flag_bnd) return fail(d, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
    const Cls& k = plan[class_of[p]];
    if (x_out && x_out[p])
      memcpy(x_out[p], hsol + k.sol + (size_t)slot_of[p] * k.npad, (size_t)3 * probs[p]->mesh.nbe * sizeof(double2));
  }
  if (corr_out) {
    // class norms were staged at the class's first sorted position
    for (int p = 0; p < nprob; ++p) {
      if (!(mixed && iters > 0)) {
        corr_out[p] = 0.0;
        continue;
      }
      const Cls& k = plan[class_of[p]];
      const int B = k.g1 - k.g0;
      const unsigned long long* hn = hnorm + (size_t)2 * (kMaxRefine + 1) * k.g0 + (size_t)2 * B * (iters - 1);
      double dm, xm;
      memcpy(&dm, &hn[2 * slot_of[p]], sizeof dm);
      memcpy(&xm, &hn[2 * slot_of[p] + 1], sizeof xm);
      corr_out[p] = xm > 0 ? dm / xm : 0.0;
    }
  }
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// Serving slots: one problem per context, kept on the device after its solve
// (FP64 H, its factors and the post-swap G), so that a new right-hand side for
// the same (mesh, material, omega, KODE) costs a GEMV and the refinement.
// ---------------------------------------------------------------------------
size_t slot_footprint(int nn, int nbe, int ng, bool mixed) {
  const size_t lda = (size_t)((nn + 1) & ~1), a_stride = lda * (size_t)(nn + 1);
  const int jc = std::max(1, std::min(64, 1024 / std::max(ng, 1)));
  const size_t chunks = (size_t)(nbe + jc - 1) / jc;
  const size_t resid_chunks = (size_t)(nn + kResidCols - 1) / kResidCols;
  size_t b = a_stride * sizeof(double2) * 2;               // A64 and G64
  if (mixed) b += a_stride * sizeof(float2);               // A32
  b += (size_t)nn * (sizeof(double2) + sizeof(float2));   // x64, v32
  b += resid_chunks * nn * sizeof(double2);                // residual partials
  b += (size_t)nbe * 9 * 2 * sizeof(double2);              // diagonal blocks
  b += chunks * nn * sizeof(double2);                      // RHS partials
  b += (size_t)nn * (sizeof(int) + 2 * sizeof(double2));   // pivots, solve scratch
  if (mixed) b += (size_t)(2 * nn + 2 * (nn + 1)) * 64 * sizeof(float);  // tensor-core operands
  return b;
}

int slot_solve_full(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                    double fr, bool mixed, int iters) {
  if (iters < 0 || iters > kMaxRefine) return fail(ctx, BEM_ERR_ARG, "refinement steps out of range");
  int rc = ensure_sweep(ctx, 1, mixed, true);
  if (rc) return rc;
  SweepBuf& S = ctx->sweep;
  const int nn = S.nn;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  DynBatch db{};
  db.zge = zge;
  db.zcs = zcs;
  db.zcp = zcp;
  db.c = c;
  db.freqs = &fr;
  db.batch = 1;
  db.flags = BEM_FAST_SINGULAR;
  db.A = S.A64;
  db.lda = S.lda;
  db.a_stride = S.a_stride;
  db.A32 = mixed ? S.A32 : nullptr;
  db.diag_h = S.diag_h;
  db.diag_g = S.diag_g;
  db.rhs_part = S.rhs_part;
  db.G = S.G64;
  rc = launch_dynamic_batch(ctx, db);
  if (rc) return rc;
  if (!mixed) return lu_factor_solve_batch(ctx, S.A64, S.lda, S.a_stride, nn, 1, false);
  rc = lu_factor_solve_batch(ctx, S.A32, S.lda, S.a_stride, nn, 1, true);
  if (rc) return rc;
  k_x_init<<<(nn + 255) / 256, 256, 0, ctx->stream>>>(S.A32, S.lda, S.a_stride, nn, S.x64, nn);
  ctx->launches++;
  BEM_CUDA(ctx, cudaMemsetAsync(S.norm, 0, (size_t)2 * (kMaxRefine + 1) * sizeof(unsigned long long),
                                ctx->stream));
  return refine_steps(ctx, S, 1, iters, 0);
}

int slot_solve_rhs(bem_ctx* ctx, bool mixed, int iters) {
  SweepBuf& S = ctx->sweep;
  if (!S.G64 || !ctx->zdfi) return fail(ctx, BEM_ERR_STATE, "no cached problem on this context");
  if (iters < 0 || iters > kMaxRefine) return fail(ctx, BEM_ERR_ARG, "refinement steps out of range");
  const int nn = S.nn;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  // b = G ZDFI (FP64): into column nn of A64 (the refinement's b), or into x64
  // for the FP64 triangular solves.
  k_resid_partial<<<dim3((nn + kResidRows - 1) / kResidRows, S.resid_chunks, 1), kResidRows, 0, ctx->stream>>>(
      S.G64, S.lda, S.a_stride, ctx->zdfi, 0, nn, S.resid_chunks, S.part);
  double2* b = mixed ? S.A64 + (size_t)nn * S.lda : S.x64;
  k_gemv_final<<<(nn + 255) / 256, 256, 0, ctx->stream>>>(S.part, nn, S.resid_chunks, b);
  ctx->launches += 2;
  BEM_CUDA(ctx, cudaGetLastError());
  if (!mixed) return lu_solve_vec(ctx, S.A64, S.lda, S.a_stride, nn, 1, S.x64, nn, false);
  // x = 0, then one more step than requested: the first one is the FP32 solve.
  BEM_CUDA(ctx, cudaMemsetAsync(S.x64, 0, (size_t)nn * sizeof(double2), ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(S.norm, 0, (size_t)2 * (kMaxRefine + 1) * sizeof(unsigned long long),
                                ctx->stream));
  return refine_steps(ctx, S, 1, iters + 1, 0);
}

// Serving batches: `batch` frequencies of the resident mesh with the same
// boundary conditions in lockstep (one assembly launch, one lockstep LU and
// refinement), as one step of bem_sweep; not kept for right-hand-side reuse.
int slot_solve_batch(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                     const double* freqs, int batch, bool mixed, int iters) {
  if (iters < 0 || iters > kMaxRefine) return fail(ctx, BEM_ERR_ARG, "refinement steps out of range");
  if (batch < 1 || batch > kMaxBatch) return fail(ctx, BEM_ERR_ARG, "batch size out of range");
  int rc = ensure_sweep(ctx, batch, mixed, false);
  if (rc) return rc;
  SweepBuf& S = ctx->sweep;
  const int nn = S.nn;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  DynBatch db{};
  db.zge = zge;
  db.zcs = zcs;
  db.zcp = zcp;
  db.c = c;
  db.freqs = freqs;
  db.batch = batch;
  db.flags = BEM_FAST_SINGULAR;
  db.A = S.A64;
  db.lda = S.lda;
  db.a_stride = S.a_stride;
  db.A32 = mixed ? S.A32 : nullptr;
  db.diag_h = S.diag_h;
  db.diag_g = S.diag_g;
  db.rhs_part = S.rhs_part;
  rc = launch_dynamic_batch(ctx, db);
  if (rc) return rc;
  if (!mixed) return lu_factor_solve_batch(ctx, S.A64, S.lda, S.a_stride, nn, batch, false);
  rc = lu_factor_solve_batch(ctx, S.A32, S.lda, S.a_stride, nn, batch, true);
  if (rc) return rc;
  k_x_init<<<dim3((nn + 255) / 256, batch), 256, 0, ctx->stream>>>(S.A32, S.lda, S.a_stride, nn, S.x64, nn);
  ctx->launches++;
  BEM_CUDA(ctx, cudaMemsetAsync(S.norm, 0, (size_t)2 * batch * (kMaxRefine + 1) * sizeof(unsigned long long),
                                ctx->stream));
  return refine_steps(ctx, S, batch, iters, 0);
}

// Raw solution of problem b of the last slot_solve_batch.
const double2* slot_batch_solution(bem_ctx* ctx, bool mixed, int b) {
  SweepBuf& S = ctx->sweep;
  if (mixed) return S.x64 + (size_t)b * S.nn;
  return S.A64 + (size_t)b * S.a_stride + (size_t)S.nn * S.lda;
}

const double2* slot_solution(bem_ctx* ctx, bool mixed, bool rhs_only) {
  SweepBuf& S = ctx->sweep;
  if (mixed || rhs_only) return S.x64;
  return S.A64 + (size_t)S.nn * S.lda;
}

}  // namespace bem
