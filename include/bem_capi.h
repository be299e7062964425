/*
 * bem_capi.h -- C-ABI of libbem_b200.so, the B200 (sm_100a) implementation
 * of the BEM-MECECCS hot path: H/G assembly (GHMATECE/GHMATECD) and the
 * dense complex solve (LINSOLVE).
 *
 * Two layers:
 *
 *  1. The drop-in seam.  The exact gfortran-mangled entry points that the
 *     reference's Fortran driver calls when built with -DUSE_GPU (lower case
 *     plus '_', every argument by reference, no hidden lengths).  A Fortran
 *     build of the reference links against this library instead of its own
 *     CUDA sources under src/kernels/.  FP64 form only (FREAL=double, COMPLEX = 16-byte
 *     interleaved re/im, INTEGER = int32).  State lives in one process-wide
 *     context, like the reference's device globals (src/kernels/shared.cu:6-31).
 *     Errors follow the reference: *status = 1 on a degenerate Jacobian, and
 *     CUDA / solver failures print a message and exit(1).
 *
 *  2. The native API (bem_*).  An explicit context per mesh, status codes
 *     instead of exit(), device-resident state that can be kept across
 *     frequencies, and an optional caller stream.  A context's device memory
 *     comes from the device's stream-ordered pool (cudaMallocAsync on the
 *     context's stream; the pool keeps freed memory for later contexts), so
 *     destroying a context does not synchronise the rest of the device.
 *
 * Layouts follow the reference (Fortran column-major):
 *   cone[k*n + i]            CONE(i+1,k+1), 1-based node numbers, n x 4
 *   etas[3*j + c]            ETAS(c+1,j+1)
 *   hestdiag[9*a + 3*j + i]  HESTdiag(i+1,j+1,a+1)  (same for gestdiag)
 *   zh[col*nn + row]         ZH(row+1,col+1), nn = 3*nbe, complex interleaved
 */
#ifndef BEM_CAPI_H
#define BEM_CAPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* 1. Drop-in seam (gfortran name mangling, all arguments by reference).     */
/* ------------------------------------------------------------------------ */

/* Replaces send_shared_data_to_gpu_, src/kernels/shared.cu:84-99.
 * Uploads the mesh and the Gauss rule; precomputes Gauss-point geometry. */
void send_shared_data_to_gpu_(double cx[], double cy[], double cz[],
                              double cxm[], double cym[], double czm[],
                              double etas[], double gi[], double ome[],
                              int cone[], int *np, int *npg, int *n, int *nbe);

/* Replaces send_dyn_data_gpu_, src/kernels/shared.cu:168-182.
 * zdfi: 3*nbe complex (re,im pairs); kode: 3*nbe. */
void send_dyn_data_gpu_(int *nbe, double zdfi[], int kode[]);

/* Replaces cuda_ghmatece_, src/kernels/Ghmatece_cu.cu:264-371.
 * Static Kelvin T over NBE x N element pairs with the rigid-body row sum
 * fused; HESTdiag stays on the device (hestdiag is not written, as in the
 * reference without TEST_CUDA).  *status = 1 on DET < 1e-5. */
void cuda_ghmatece_(int *nbe, int *npg, int *n, int *np, double *c3,
                    double *c4, double *fr, double hestdiag[], int *status);

/* Replaces cuda_send_gest_data_, src/kernels/Ghmatece_cu.cu:373-380.
 * Uploads the CPU-computed GESTdiag (3,3,NBE). */
void cuda_send_gest_data_(int *nbe, double *gestdiag);

/* Replaces cuda_ghmatecd_, src/kernels/Ghmatecd_cu.cu:305-483.
 * Assembles ZH with the boundary-condition column swap applied and the
 * right-hand side ZFI = ZG*ZDFI on the device; both stay there for
 * cuda_linsolve_ (zfi and zhp are not written, as in the reference without
 * TEST_CUDA).  fast_singular = 1 integrates Stokes minus Kelvin on the
 * diagonal and adds the static diagonals.  *status = 1 on DET < 1e-5. */
void cuda_ghmatecd_(int *nbe, int *npg, int *n, int *np, double zge[2],
                    double zcs[2], double zcp[2], double *c1, double *c2,
                    double *c3, double *c4, double *fr, double hestdiag[],
                    double gestdiag[], double zfi[], double zhp[],
                    int kode[], int *fast_singular, int *status);

/* Replaces cuda_linsolve_, src/kernels/Linsolve_cu.cu:53-126.
 * LU with partial pivoting of the device-resident ZH and solve for ZFI;
 * copies the solution into zfi (nn complex).  zh is not read.  A singular
 * matrix prints an error and exits, as the reference's lu_assert does. */
void cuda_linsolve_(int *nn, int *n, double zh[], double zfi[]);

/* Replaces cuda_interec1_, src/kernels/Interec1_cu.cu:44-237 (interface
 * src/kernels/Interec1_cu.fd; caller src/Interec.for:142-164).  Displacements
 * at the l interior points (cxi, cyi, czi) from the boundary displacements
 * zfi and tractions zdfi (3*nbe complex each, after INTEREC's un-swap):
 * zdsol (3*l complex).  c1..c4 are unused, as in the reference.
 * *status = 1 on DET < 1e-5. */
void cuda_interec1_(int *n, int *nbe, int *npg, int *l, int *np, double cxi[],
                    double cyi[], double czi[], double zge[2], double zcs[2],
                    double zcp[2], double *c1, double *c2, double *c3,
                    double *c4, double *fr, double zdfi[], double zfi[],
                    double zdsol[], int *status);

/* Replaces deallocate_shared_gpu_data_, src/kernels/shared.cu:184-214. */
void deallocate_shared_gpu_data_(void);

/* ------------------------------------------------------------------------ */
/* 2. Native API.                                                            */
/* ------------------------------------------------------------------------ */

enum bem_status {
  BEM_OK = 0,
  BEM_ERR_DEGENERATE = 1, /* DET < 1e-5 at some Gauss point */
  BEM_ERR_SINGULAR = 2,   /* zero pivot in the LU */
  BEM_ERR_ARG = 3,        /* bad argument or size */
  BEM_ERR_CUDA = 4,       /* CUDA runtime error */
  BEM_ERR_NOMEM = 5,      /* device allocation failed */
  BEM_ERR_STATE = 6,      /* call out of order (e.g. solve before assembly) */
  BEM_ERR_TIMEOUT = 7     /* a bounded device-side wait gave up */
};

typedef struct bem_ctx bem_ctx;

/* Flags of bem_ghmatecd. */
#define BEM_FAST_SINGULAR 1  /* the reference's fast_singular = 1 */
#define BEM_KEEP_PRESWAP 2   /* also keep pre-swap H and G for read-back */

int bem_ctx_create(int device, bem_ctx **out);
int bem_ctx_destroy(bem_ctx *ctx);
/* Runs every kernel of ctx on `stream` (a cudaStream_t); NULL restores the
 * context's own stream. */
int bem_ctx_set_stream(bem_ctx *ctx, void *stream);
/* Algorithm switches of a context (1 on, 0 off), for comparison and for the
 * autotuner: "tcgen05" (FP32 trailing update on tcgen05, else TF32
 * mma.sync), "trsv_coop" (one cooperative launch per triangular solve),
 * "lu_pairs" (two 64-column panels per FP32 trailing update, K = 128),
 * "lu_quads" (four, K = 256, where they fit), "f64_cublas" (FP64 LU: the
 * trailing update by cuBLAS ZGEMM, one panel per update; the plain FP64
 * form's library GEMM), "f64_pairs" (FP64 LU with f64_cublas off: two
 * panels per trailing update on the DMMA kernel, K = twice the panel
 * width), "tc_pair" (the FP32
 * trailing update by CTA pairs on tcgen05 cta_group::2, M = 256 per pair),
 * "small_clusters" (panel clusters of 2, 4 or 8 CTAs for systems whose
 * panel rows fit them at <= 256 rows per CTA, instead of always 16),
 * "panel_tslu" (FP32 panels taller than a 16-CTA cluster holds, about 6900
 * rows: tournament pivoting over cluster-sized chunks instead of the
 * grid-barrier kernel),
 * "panel_calu" (FP32 panels with
 * tournament pivoting), "panel_push" (cluster panels push their pivot
 * candidates by remote stores), "panel_async" (... as st.async into
 * mbarrier-counted mailboxes, without a cluster barrier per column),
 * "laswp_tc" (FP32 row interchanges + U12 on the tensor cores), "trsv_inv"
 * (FP32 solves with inverted diagonal blocks), "graphs" (bem_sweep replays a
 * captured step).  Defaults: tcgen05, tc_pair, trsv_coop, lu_pairs,
 * lu_quads, f64_cublas, f64_pairs, small_clusters, panel_push, panel_async,
 * laswp_tc, trsv_inv and graphs on; panel_calu and panel_tslu off (measured
 * no faster on B200).
 * Integer budgets for a context that shares the GPU with another one running
 * at the same time (0, the default, means the whole device): "gemm_ctas"
 * (CTAs of the persistent FP32 trailing update) and "trsv_ctas" (CTAs of one
 * cooperative triangular solve, over all problems of the batch).
 * "wait_limit_ms" (1..60000, default 2000): how long any device-side wait of
 * ctx's kernels (a bulk-copy mbarrier, a cluster mailbox, a software grid
 * barrier) may last before the kernel gives up, records a timeout and
 * returns; the call then reports BEM_ERR_TIMEOUT. */
int bem_ctx_set_option(bem_ctx *ctx, const char *name, int value);
int bem_ctx_get_option(bem_ctx *ctx, const char *name, int *value);
const char *bem_status_string(int status);
const char *bem_last_error(bem_ctx *ctx);
/* Number of kernels this library launched on ctx since creation. */
long long bem_ctx_launch_count(bem_ctx *ctx);

/* Mesh upload, as send_shared_data_to_gpu_. */
int bem_mesh_upload(bem_ctx *ctx, int n, int nbe, int np, int npg,
                    const int *cone, const double *cx, const double *cy,
                    const double *cz, const double *cxm, const double *cym,
                    const double *czm, const double *etas, const double *gi,
                    const double *ome);

/* GHMATECE on the device.  c = {C1,C2,C3,C4} (src/Ghmatece.for:60-63).
 * Computes HESTdiag (rigid body) and, if compute_gest, GESTdiag (SINGGE on
 * the device).  Outputs may be NULL; results stay resident. */
int bem_ghmatece(bem_ctx *ctx, const double c[4], int compute_gest,
                 double *hestdiag_out, double *gestdiag_out);

/* Upload host static diagonals (cuda_send_gest_data_ and its H twin). */
int bem_set_gestdiag(bem_ctx *ctx, const double *gestdiag);
int bem_set_hestdiag(bem_ctx *ctx, const double *hestdiag);

/* Full static H (3nbe x 3n, column-major) for checking; may be slow. */
int bem_static_h(bem_ctx *ctx, const double c[4], double *hest_out);

/* Boundary conditions, as send_dyn_data_gpu_. zdfi: 3nbe complex. */
int bem_dyn_upload(bem_ctx *ctx, const double *zdfi, const int *kode);

/* GHMATECD on the device: swapped ZH and RHS ZFI assembled in place. */
int bem_ghmatecd(bem_ctx *ctx, const double zge[2], const double zcs[2],
                 const double zcp[2], const double c[4], double fr,
                 int flags);

/* Read back the assembled system: zh nn x nn (after the swap), zfi nn.
 * Either may be NULL.  Valid after bem_ghmatecd, before bem_linsolve. */
int bem_get_system(bem_ctx *ctx, double *zh, double *zfi);
/* Pre-swap H and G (needs BEM_KEEP_PRESWAP at assembly). */
int bem_get_preswap(bem_ctx *ctx, double *zh, double *zg);

/* GHMATECD that allocates nothing.  No counterpart in the reference: it is an
 * addition for callers that must not allocate device memory once set up --
 * a serving process that has handed its free HBM to its own pool or cache
 * (bem_ghmatecd would add a 16 nn^2-byte system behind its back), or a loop
 * that cannot afford cudaFree's device-wide synchronisation.
 * Same assembly as bem_ghmatecd (flags: 0 or BEM_FAST_SINGULAR), written to
 * the caller's device buffer a: nn x (nn + 1) complex128, column-major with
 * leading dimension lda >= nn (complex elements), 16-byte aligned; columns
 * 0..nn-1 receive ZH after the BC swap, column nn the RHS ZFI -- the values
 * bem_get_system returns.  ctx's own system is left untouched.  The
 * assembly's scratch (2 x 9 nbe + chunks x nn complex128 words, chunks =
 * ceil(nbe / min(64, 1024 / npg^2))) comes from one fixed 8 MiB array that
 * each device holds until the process exits; a larger mesh is rejected with
 * BEM_ERR_ARG (nbe <= 3136 at npg <= 4, 2520 at 5, 2128 at 6, 1801 at 7, 1618 at
 * npg = 8).  The first call on a device looks up that array's device address
 * and keeps it for the life of the process; make it before any stream
 * capture.  The kept address does not survive cudaDeviceReset on that device:
 * after a reset this entry point must not be called again in the process.
 * All calls on a device share the array: calls that overlap on the GPU
 * (other streams, other contexts of the same device) race.  Asynchronous on
 * ctx's stream; a device-side timeout shows at the next bem_sync. */
int bem_ghmatecd_noalloc(bem_ctx *ctx, const double zge[2],
                         const double zcs[2], const double zcp[2],
                         const double c[4], double fr, int flags, double *a,
                         size_t lda);

/* LINSOLVE on the device: factor the assembled ZH, solve for ZFI, copy the
 * solution (nn complex) to zfi_out (may be NULL to keep it on the device). */
int bem_linsolve(bem_ctx *ctx, double *zfi_out);

/* ZGESV on the device for one right-hand side (src/Linsolve.for:94-100):
 * a is nn x nn column-major complex (host), b nn complex (host); the
 * solution is written to x (host).  Uses the same LU as bem_linsolve and
 * replaces any assembled system of ctx. */
int bem_solve_dense(bem_ctx *ctx, int nn, const double *a, const double *b,
                    double *x);

/* Static boundary solve.  No counterpart in the reference (it keeps only
 * HESTdiag and GESTdiag of the static problem); an extension built from its
 * static pieces: H = Kelvin T off the diagonal (NONSINGE) + HESTdiag, G =
 * Kelvin U off the diagonal (NONSINGE_G / SOLFUNE_G, Singge.for:83-202) +
 * GESTdiag, the boundary-condition swap with the real GE, G*dfi, the FP64 LU
 * of bem_linsolve and the un-swap.  c = {C1..C4} of the static material
 * (the ones bem_ghmatece was called with), kode/dfi: 3*nbe; disp/trac:
 * 3*nbe real.  Replaces any assembled system of ctx. */
int bem_static_solve(bem_ctx *ctx, const double c[4], double ge,
                     const int *kode, const double *dfi, double *disp,
                     double *trac);

/* The Interec.for:59-67 un-swap of the last solution: boundary
 * displacements into disp_out and tractions into trac_out (nn complex). */
int bem_unswap(bem_ctx *ctx, double *disp_out, double *trac_out);

/* Synchronise ctx's stream; returns the first pending error. */
int bem_sync(bem_ctx *ctx);

/* bem_linsolve without the read-back and without synchronising: the
 * factorisation and solve are only enqueued on ctx's stream; errors are
 * reported by the next bem_sync. */
int bem_linsolve_async(bem_ctx *ctx);

/* Frequency sweep on the resident mesh (the batching and precision forms).
 * Assembles and solves nfreq frequencies, `batch` (1..64) problems at a
 * time in lockstep.  form BEM_FORM_PLAIN: FP64 assembly and FP64 LU.
 * form BEM_FORM_MIXED: FP64 assembly plus a complex64 copy, FP32 LU with
 * TF32 tensor-core updates, then `refine` (0..8) steps of FP64 iterative
 * refinement against the FP64 matrix.  `batch` is an upper bound: no more
 * problems run in lockstep than bem_sweep_batch_limit reports, so that every
 * problem's panel factorisation runs in the same wave (results do not depend
 * on the grouping).  x_out (nfreq x nn complex, may be
 * NULL) receives the raw solutions (before the un-swap); corr_out (nfreq,
 * may be NULL) the relative size max|d|/max|x| of the last refinement
 * correction.  With both NULL the call only enqueues work on ctx's stream. */
#define BEM_FORM_PLAIN 0
#define BEM_FORM_MIXED 1
int bem_sweep(bem_ctx *ctx, const double zge[2], const double zcs[2],
              const double zcp[2], const double c[4], const double *freqs,
              int nfreq, int form, int batch, int refine, double *x_out,
              double *corr_out);

/* bem_sweep that returns once its work and the copies of its solutions into
 * x_out are enqueued on ctx's stream (no corrections).  x_out should be
 * page-locked host memory (or device memory) for the copies to overlap; it
 * must stay untouched until the stream has passed them: record an event on
 * the stream given to bem_ctx_set_stream, or call bem_sync, which also
 * reports the errors of this call.  A client keeps several sweeps of one
 * context in flight this way, each into its own output buffer. */
int bem_sweep_async(bem_ctx *ctx, const double zge[2], const double zcs[2],
                    const double zcp[2], const double c[4],
                    const double *freqs, int nfreq, int form, int batch,
                    int refine, double *x_out);

/* Many problems of uneven size in lockstep (the batching form for small
 * meshes).  probs[p] is a context holding problem p's mesh, static
 * diagonals (bem_ghmatece) and BCs (bem_dyn_upload); p is solved at
 * freqs[p] with material zge/zcs/zcp[2p..2p+1] and static constants
 * c[4p..4p+3].  The problems are sorted by size and grouped into classes
 * (largest <= 1.25 x smallest, at most bem_sweep_batch_limit problems); each
 * class is assembled into one padded size (the problem, then the identity,
 * which never pivots) and factored, solved and -- form BEM_FORM_MIXED --
 * refined together, on the driver context's stream and workspaces.  x_out[p]
 * (3 nbe_p complex, raw as bem_sweep's; NULL entries skipped) and corr_out[p]
 * (may be NULL) receive the results.  Synchronous.  No counterpart in the
 * reference (its driver solves one mesh at a time). */
int bem_batch_solve(bem_ctx *driver, int nprob, bem_ctx *const *probs,
                    const double *freqs, const double *zge, const double *zcs,
                    const double *zcp, const double *c, int form, int refine,
                    double *const *x_out, double *corr_out);

/* Largest lockstep batch bem_sweep uses for this mesh and form: the number
 * of panel-factorisation thread-block clusters the device keeps resident at
 * once (7 for n = 6480 on a 148-SM B200), capped at 64. */
int bem_sweep_batch_limit(bem_ctx *ctx, int form, int *limit);

/* Kernel-class timing with CUDA events on ctx's stream.  Classes:
 * 0 assembly, 1 LU panel, 2 row interchange + triangular solve,
 * 3 trailing-update GEMM, 4 back substitution and refinement solves,
 * 5 refinement residual.  work[c] is the algorithmic work of the class:
 * Stokes evaluations for 0, real flops for 3 (8 m n k per complex update)
 * and 5 (8 n^2 per residual), 0 otherwise. */
#define BEM_PROF_CLASSES 6
int bem_prof_enable(bem_ctx *ctx, int on);
int bem_prof_reset(bem_ctx *ctx);
int bem_prof_read(bem_ctx *ctx, double *ms, long long *launches,
                  double *work);
/* Algorithmic device-memory bytes per class since the last reset (data each
 * class must read or write at least once: the panel slices, the rows
 * interchanged and solved, C read and written once per trailing update, the
 * factors read once per solve, the FP64 matrix once per residual, the
 * systems written by the assembly). */
int bem_prof_bytes(bem_ctx *ctx, double *bytes);

/* Failure-path self-test.  No counterpart in the reference (its CUDA waits
 * are unbounded): runs one small kernel with the library's bounded wait of
 * kind `which` on an event that never happens -- 0: an mbarrier armed for a
 * bulk copy that is never issued; 1: a software grid barrier that expects one
 * CTA more than the launch has -- under ctx's "wait_limit_ms".  The kernel
 * gives up after that limit and returns, and the call reports
 * BEM_ERR_TIMEOUT; ctx stays usable (the next call clears the status).
 * Nothing faults or hangs. */
int bem_wait_selftest(bem_ctx *ctx, int which);

/* Measures this GPU's FP64 tensor-core (DMMA) throughput with a
 * register-resident mma.sync loop; writes TFLOP/s. */
int bem_measure_fp64_peak(bem_ctx *ctx, double *tflops);

/* INTEREC's interior part on the device (src/Interec.for:81-285): for l
 * interior points (cxi, cyi, czi), the displacements zdsol (3*l complex,
 * NONSINGD as in src/Interec.for:111-133) and, when zssol is not NULL, the
 * stresses zssol (9*l complex, SIGMAEC src/Sigmaec.for:9-212 contracted as in
 * src/Interec.for:188-283; component (i, j) at 9k + i + 3j), from the
 * boundary displacements `disp` and tractions `trac` (3*nbe complex each,
 * after the un-swap, e.g. from bem_unswap).  rho is the density (stresses
 * only).  Synchronous. */
int bem_interior(bem_ctx *ctx, const double zge[2], const double zcs[2],
                 const double zcp[2], double rho, double fr, int l,
                 const double *cxi, const double *cyi, const double *czi,
                 const double *disp, const double *trac, double *zdsol,
                 double *zssol);

/* ------------------------------------------------------------------------ */
/* 3. Serving (no counterpart in the reference: its driver solves one mesh   */
/*    at a time).                                                             */
/* ------------------------------------------------------------------------ */

/* A request loop on one GPU.  Requests (mesh, material, omega, boundary
 * conditions) are solved as they arrive: a scheduler thread admits every
 * request that fits `budget_bytes` of device memory into a slot (one problem
 * with its own stream and workspaces) and enqueues it at once, so requests
 * that arrive while others run overlap with them on the device.  A solved
 * problem stays resident (H, its factors and the post-swap G): a later
 * request with the same mesh, material, omega and KODE but a new right-hand
 * side is solved with the cached factors (GEMV + solves).  Idle problems are
 * evicted least-recently-used when a new one needs room.  Queued requests
 * with the same mesh, material, boundary values and KODE (a sweep over omega)
 * are solved together as one lockstep batch.  At most 8 slots and 16
 * problems are in flight at once (more would only queue their kernels behind
 * each other on the GPU); a request that fits the budget waits.  form:
 * BEM_FORM_PLAIN or BEM_FORM_MIXED (with `refine` refinement steps). */
typedef struct bem_server bem_server;
int bem_server_create(int device, double budget_bytes, int form, int refine,
                      bem_server **out);
int bem_server_destroy(bem_server *srv);
/* Registers a mesh (the arrays of bem_mesh_upload, copied); returns its id. */
int bem_server_add_mesh(bem_server *srv, int n, int nbe, int np, int npg,
                        const int *cone, const double *cx, const double *cy,
                        const double *cz, const double *cxm, const double *cym,
                        const double *czm, const double *etas,
                        const double *gi, const double *ome, int *mesh_id);
/* material = {GE, nu, damping, density} (Inputecd.for:58-60); bc: 3*nbe
 * complex (ZDFI), kode: 3*nbe.  Returns at once with a request id. */
int bem_server_submit(bem_server *srv, int mesh_id, const double material[4],
                      double fr, const double *bc, const int *kode,
                      long long *req_id);
/* Waits up to timeout_s for a request; on BEM_OK writes the boundary
 * displacements and tractions (3*nbe complex each, after the un-swap) and
 * info = {latency ms (submit to done), queueing ms (submit to start),
 * 1 if solved with cached factors, device bytes of its slot}.  Returns the
 * request's status (BEM_ERR_TIMEOUT if still running; the request then
 * stays waitable).  A request is forgotten once waited for. */
int bem_server_wait(bem_server *srv, long long req_id, double timeout_s,
                    double *disp, double *trac, double *info);
/* out[10] = {completed, p50 ms, p99 ms, solves/s (completed / time from the
 * first submit to the last completion), cached-factor solves, evictions,
 * peak admitted bytes, most slots busy at once, admitted bytes now,
 * budget}. */
int bem_server_stats(bem_server *srv, double *out);
int bem_server_reset_stats(bem_server *srv);

/* Microbenchmarks of the arithmetic peaks this library's rooflines use,
 * TFLOP/s, in out[5]: FP64 FMA, FP32 FMA (SIMT, 8 independent chains per
 * thread), FP64 DMMA m8n8k4, tcgen05 kind::tf32 with M=128 and N=128, and
 * with N=256 (operands in shared memory, accumulator in TMEM). */
int bem_measure_peaks(bem_ctx *ctx, double *out);

#ifdef __cplusplus
}
#endif
#endif /* BEM_CAPI_H */
