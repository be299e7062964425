// bem_internal.h -- the context behind the C-ABI and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "bem_capi.h"
#include "bem_device.cuh"

namespace bem {

// Largest Gauss rule per direction (the reference's fixtures use 8).
constexpr int kMaxNpg = 8;
// Largest number of problems assembled or factored in lockstep.
constexpr int kMaxBatch = 64;
// Largest number of iterative-refinement steps of the mixed form.
constexpr int kMaxRefine = 8;

// Device buffers of bem_sweep (per batch of problems).
struct SweepBuf {
  int nn = 0, batch = 0, rhs_chunks = 0, resid_chunks = 0;
  size_t lda = 0, a_stride = 0;
  double2* A64 = nullptr;       // [batch] x nn x (nn+1)
  float2* A32 = nullptr;        // complex64 copies (mixed form)
  double2* x64 = nullptr;       // [batch][nn] refined solutions
  float2* v32 = nullptr;        // [batch][nn] refinement right-hand sides
  double2* part = nullptr;      // [batch][resid_chunks][nn] residual partials
  double2 *diag_h = nullptr, *diag_g = nullptr;  // [batch][nbe][9]
  double2* rhs_part = nullptr;  // [batch][rhs_chunks][nn]
  unsigned long long* norm = nullptr;  // [kMaxRefine][batch][2] max|d|, max|x|
  double2* G64 = nullptr;       // [batch] post-swap G (serving: right-hand-side reuse)
  size_t norm_cap = 0;          // problems the norm buffer holds (batched solves)
};

// One batched dynamic assembly: `batch` frequencies of the resident mesh.
struct DynBatch {
  const double *zge, *zcs, *zcp, *c;
  const double* freqs;
  int batch, flags;
  double2* A;          // problem b at A + b*a_stride
  size_t lda, a_stride;
  float2* A32;         // optional complex64 copy, same layout
  double2 *zh_pre, *zg_pre;
  double2 *diag_h, *diag_g;  // [batch][nbe][9]
  double2* rhs_part;         // [batch][chunks][nn]
  double2* G = nullptr;      // optional post-swap G, same layout as A
};

struct Mesh {
  int n = 0, nbe = 0, np = 0, npg = 0, ng = 0;  // ng = npg^2
  double4* gq = nullptr;      // [n][ng] Gauss point (x, y, z, w1*w2*det)
  double4* eta = nullptr;     // [n] unit normal (x, y, z, 0)
  double4* colloc = nullptr;  // [n] collocation point = centroid
  double* corner = nullptr;   // [n][12] corner coordinates CO(4,3) row-major
  int* degen = nullptr;       // [n] 1 when some DET < 1e-5 on the element
  double gi[kMaxNpg], ome[kMaxNpg];
};

struct System {
  int nn = 0;              // 3 * nbe
  size_t lda = 0;          // leading dimension of A
  double2* A = nullptr;    // nn x (nn + 1): ZH after the swap | RHS column
  double2* zh_pre = nullptr, *zg_pre = nullptr;  // optional pre-swap copies
  double2* diag_h = nullptr, *diag_g = nullptr;  // [nbe][9] pre-swap diagonal blocks
  double2* rhs_part = nullptr;                   // [chunks][nn]
  int rhs_chunks = 0;
  double2* x = nullptr;        // [nn] solution (raw, before the un-swap)
  double2* zdfi_last = nullptr;  // [nn] right-hand data used by the last assembly
  double2 zge_last = {0, 0};
  bool assembled = false, solved = false, have_preswap = false;
};

// Gather list of one panel's row interchanges: count, then dst/src pairs.
constexpr int kPermStride = 1 + 2 * 128;

struct LuWork {
  int cap_nn = 0, cap_batch = 0;
  int cluster_cs = 0;           // CTAs per panel cluster (16 or 8)
  int* ipiv = nullptr;          // [batch][nn] 1-based pivot rows
  int* perm = nullptr;          // [panel][batch][kPermStride]
  std::vector<std::pair<int, int>> panels;  // (k, w) of every panel of the last factorisation
  double* slot_val = nullptr;   // grid-panel fallback: [2][kMaxGrid]
  int* slot_row = nullptr;      // [2][kMaxGrid]
  double2* cand = nullptr;      // [2][kMaxGrid][64]
  double2* drow = nullptr;      // [2][64]
  unsigned* barrier = nullptr;  // grid barrier counter
  // cooperative triangular solves (k_trsv)
  void* trsv_w = nullptr;       // [batch][2][nn] scratch vectors
  size_t trsv_w_bytes = 0;
  unsigned* trsv_ctr = nullptr;  // [kMaxBatch] group barrier counters
  int* pstart = nullptr;         // first row of each panel of the last factorisation, then nn
                                 // (written by the panel kernels)
  float2* linv = nullptr;        // [batch][64][64] L11^-1 of the current FP32 panel (k_laswp_tc)
  size_t linv_bytes = 0;
  int* gmap = nullptr;           // [batch][kGroupMaps][nn] row maps of a panel group (k_l11_inv)
  size_t gmap_bytes = 0;
  // tall FP32 panels by tournament (tslu_panel): chunk copies and their pivots,
  // the candidates, their row indices and pivots
  float2* ts_s = nullptr;
  int* ts_ipiv = nullptr;
  int* ts_perm = nullptr;
  float2* ts_c = nullptr;
  int* ts_gid = nullptr;
  int* ts_cipiv = nullptr;
  int* ts_cperm = nullptr;
  size_t ts_cap[7] = {0, 0, 0, 0, 0, 0, 0};  // elements allocated, in the order above
  float2* tinv = nullptr;        // FP32 solves: inverted diagonal blocks of the last factors
  size_t tinv_bytes = 0;
  bool tinv_valid = false;
  double2* lg = nullptr;         // FP64 panel pairs on cuBLAS: both panels' L, the first gathered
  size_t lg_cap = 0;             // elements
};

constexpr int kMaxGrid = 160;
constexpr int kGroupMaps = 3;  // row maps of the first three panels of a four-panel group

// Packed operands of the tensor-core FP32 trailing update (gemm_tc.cu).
struct TcWork {
  size_t lrows_cap = 0, urows_cap = 0;  // rows the operand buffers hold
  float* lhat = nullptr;  // [batch][2nn][64]  re/im rows of L21, TF32
  float* ure = nullptr;   // [batch][nn+1][64] Re U12, K-major, TF32
  float* uim = nullptr;   // [batch][nn+1][64] Im U12
  void* maps = nullptr;   // 6 TMA tensor maps (host copies, passed by value)
  int pair_clusters = 0;  // resident CTA pairs of k_gemm_tc2 (0: not yet queried)
  float2* cbase = nullptr;  // systems the C map (maps[3]) was made for
  size_t clda = 0, cbstride = 0;
  int cbatch = 0;
};

// CUDA-event timing per kernel class (off unless enabled).
struct Profiler {
  bool on = false;
  struct Rec {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  double ms[BEM_PROF_CLASSES] = {0};
  long long launches[BEM_PROF_CLASSES] = {0};
  double work[BEM_PROF_CLASSES] = {0};
  double bytes[BEM_PROF_CLASSES] = {0};  // algorithmic device-memory bytes
};

// Brackets one launch of class `cls` with events when profiling is on.
struct ProfScope {
  bem_ctx* ctx;
  int cls;
  cudaEvent_t b = nullptr;
  ProfScope(bem_ctx* c, int k, double work, double bytes = 0.0);
  ~ProfScope();
};

}  // namespace bem

struct bem_ctx {
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  std::string last_error;
  long long launches = 0;

  bem::Mesh mesh;
  bool have_mesh = false;
  double* hestdiag = nullptr;  // [nbe][9]
  double* gestdiag = nullptr;  // [nbe][9]
  bool have_hest = false, have_gest = false;
  double2* zdfi = nullptr;     // [3nbe]
  int* kode = nullptr;         // [3nbe]
  std::vector<double> h_zdfi;  // host copies for the un-swap
  std::vector<int> h_kode;
  bool have_dyn = false;
  int mesh_flag_all = 0;       // some element has DET < 1e-5
  int mesh_flag_bnd = 0;       // some boundary element has DET < 1e-5
  bool assembled_mesh = false; // the system in sys came from bem_ghmatecd
  bem::System sys;
  bem::LuWork lu;
  int* d_status = nullptr;     // [ST_COUNT]
  double* static_part = nullptr;  // [chunks][nbe][9] rigid-body partial sums
  int static_chunks = 0;
  bem::Profiler prof;
  bem::SweepBuf sweep;
  bem::TcWork tc;
  // interior-point workspace (interior.cu)
  double4* int_pts = nullptr;
  double2* int_ut = nullptr;    // [2][3nbe]: displacements, tractions
  double2* int_part = nullptr;  // [l][chunks][12]
  double2* int_out = nullptr;   // [l][12]
  size_t int_cap_l = 0, int_cap_nn = 0;
  bem::SweepBuf bbuf;  // padded systems of bem_batch_solve
  std::vector<bem_ctx*> workers;   // bem_batch_solve: contexts whose streams run classes concurrently
  void* pinned = nullptr;          // bem_batch_solve: pinned staging of descriptors, solutions, norms
  size_t pinned_bytes = 0;
  unsigned char* grp_desc = nullptr;  // bem_batch_solve: assembly descriptors on the device
  size_t grp_desc_bytes = 0;
  bool use_tcgen05 = true;  // FP32 trailing update on tcgen05 (else TF32 mma.sync)
  bool use_trsv_coop = true;
  bool trsv_inv = true;        // FP32 cooperative solves apply inverted diagonal blocks (k_trsv_f32)
  bool laswp_tc = true;        // FP32 row interchange + U12 solve on the tensor cores (k_laswp_tc)
  bool use_graphs = true;     // bem_sweep replays a captured batch step
  // the captured step of bem_sweep
  cudaGraph_t sweep_graph = nullptr;
  cudaGraphExec_t sweep_exec = nullptr;
  std::vector<cudaGraphNode_t> sweep_dyn_nodes;
  int sg_nn = 0, sg_bsz = 0, sg_mixed = 0, sg_iters = 0;
  long long sg_launches = 0;
  int sw_nn = 0, sw_bsz = 0, sw_mixed = 0, sw_iters = 0;  // shape of the last directly enqueued step
  bool panel_calu = false;    // FP32 LU panels: tournament pivoting per 8-column sub-panel
  bool panel_push = true;     // cluster panels exchange pivots by remote stores before the barrier
  bool panel_async = true;    // ... as st.async into mbarrier-counted mailboxes, no per-column cluster barrier
  bool lu_pairs = true;       // FP32 tensor-core LU: two 64-column panels per trailing update (K = 128)
  bool lu_quads = true;       // ... four (K = 256) where four 64-column panels fit
  bool f64_pairs = true;      // FP64 LU: two panels per trailing update (K = 2 x panel width)
  bool f64_cublas = true;     // FP64 LU: trailing update by cuBLAS ZGEMM (one panel per update)
  void* cublas = nullptr;     // cuBLAS handle (f64_cublas), created on first use
  void* cublas_ws = nullptr;  // its workspace (stream-ordered, so graph capture allocates nothing)
  bool tc_pair = true;        // FP32 trailing update by CTA pairs (k_gemm_tc2, tcgen05 cta_group::2)
  bool small_clusters = true; // panel clusters sized to the system (<= 256 rows per CTA), not always 16
  bool panel_tslu = false;    // FP32 panels taller than a cluster: tournament pivoting instead of the grid kernel
  // SM shares for contexts that run concurrently on one GPU (0: the whole device)
  int gemm_ctas = 0;          // CTAs of the persistent tensor-core trailing update
  int trsv_ctas = 0;          // CTAs of one cooperative triangular solve (all problems together)
  int wait_limit_ms = 2000;   // bound of every device-side wait (copy of the device word)
  std::unordered_map<long long, int> lockstep_cache;  // lu_lockstep_capacity by (size, precision)
  unsigned long long alloc_epoch = 0;  // device allocations so far (dev_alloc)
  unsigned long long sg_epoch = 0;     // alloc_epoch when the sweep step was captured
};

namespace bem {

int fail(bem_ctx* ctx, int code, const std::string& msg);
int cuda_fail(bem_ctx* ctx, cudaError_t e, const char* what);

// Device memory of a context comes from the device's stream-ordered pool,
// allocated and freed on the context's stream.  cudaFree synchronises the
// whole device, so a process that creates and drops contexts while others
// compute (the server evicting a cached problem while other requests run)
// would stall every stream on each drop; cudaFreeAsync does not.  The
// memory is ready in the order of the context's stream, which is where the
// library uses it (copies included); a context moved to another stream
// (bem_ctx_set_stream) waits for its old one first.  Every allocation also
// advances ctx->alloc_epoch: a captured sweep step names the buffers it was
// captured with and is replayed only while no buffer of the context has been
// (re)allocated since.
template <typename T>
cudaError_t dev_alloc(bem_ctx* ctx, T** p, size_t bytes) {
  ++ctx->alloc_epoch;
  return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, ctx->stream);
}
void dev_free(bem_ctx* ctx, void* p);

#define BEM_CUDA(ctx, call)                                   \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::bem::cuda_fail(ctx, e_, #call); \
  } while (0)

// Launchers (assembly.cu).
int launch_geometry(bem_ctx* ctx, const double* d_cx, const double* d_cy, const double* d_cz,
                    const int* d_cone, const double* d_etas, const double* d_cxm,
                    const double* d_cym, const double* d_czm);
int launch_static(bem_ctx* ctx, const double c[4], int compute_gest, double* hest_full);
int launch_dynamic(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2],
                   const double c[4], double fr, int flags);
// Solfund.for:29-35 constants of one frequency (assembly.cu).
StokesConsts<double> make_consts(const double zge[2], const double zcs[2], const double zcp[2], double fr);
// Interior displacements (and stresses when zssol is non-null) on the device (interior.cu).
int interior_points(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], double rho,
                    double fr, int l, const double* cxi, const double* cyi, const double* czi, const double* disp,
                    const double* trac, double* zdsol, double* zssol);
void release_interior(bem_ctx* ctx);
// Static boundary system (extension): swapped H into A (complex, imaginary
// parts 0), post-swap G into Gs (nn x nn real), column nn of A = Gs dfi.
int launch_static_system(bem_ctx* ctx, const double c[4], double ge, const int* d_kode, const double* d_dfi,
                         double2* A, size_t lda, double* Gs);
int dyn_graph_update(bem_ctx* ctx, cudaGraphExec_t exec, const std::vector<cudaGraphNode_t>& nodes,
                     const DynBatch& b);
int dyn_graph_nodes(bem_ctx* ctx, cudaGraph_t g, std::vector<cudaGraphNode_t>& out);
int launch_dynamic_batch(bem_ctx* ctx, const DynBatch& b);
void release_cublas(bem_ctx* ctx);
// A kernel's dynamic shared-memory limit is a process-wide attribute, and
// contexts in other host threads launch the same kernel with other sizes:
// the limit is only ever raised (under a lock), so no launch finds it lowered
// by another thread between setting it and launching.
cudaError_t raise_smem_limit(const void* func, size_t bytes);
// One member of a grouped assembly (bem_batch_solve).
struct GroupMember {
  bem_ctx* pc;  // the problem's context: mesh, static diagonals, BCs
  const double *zge, *zcs, *zcp, *c;
  double fr;
  double2* A;    // its padded slot (npad x (npad + 1), RHS in column npad)
  float2* A32;   // optional complex64 copy, same layout
  size_t lda;
  int npad;
  double2 *diag_h, *diag_g;  // [nbe][9] scratch
  double2* rhs_part;         // [chunks][nn] scratch
};
// Assembles and pads `count` problems in three launches on wk's stream; the
// descriptors go through h_desc (pinned, count x dyn_problem_bytes(), left
// untouched until the stream has passed) to d_desc (device, same size).
int launch_dynamic_group(bem_ctx* wk, const GroupMember* mem, int count, void* h_desc, void* d_desc);
size_t dyn_problem_bytes();
int rhs_chunks(bem_ctx* ctx);

// LU (lu.cu).
int lu_ensure_workspace(bem_ctx* ctx, int nn, int batch);
int lu_factor_solve(bem_ctx* ctx);
// Factor and solve `batch` problems A + b*bstride (elements of complex64 when
// fp32, else complex128), each nn x (nn+1) with the right-hand side last.
int lu_lockstep_capacity(bem_ctx* ctx, int nn, bool fp32);
int lu_factor_solve_batch(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch, bool fp32);
// Solves with the factors of the last lu_factor_solve_batch for right-hand
// sides v + b*vstride (overwritten by the solutions).
int lu_solve_vec(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch, void* v, size_t vstride,
                 bool fp32);

// Frequency sweep (mixed.cu).
// wait_out: with x_out, return once the solutions are in host memory (else
// their copies are only enqueued and errors wait for the next bem_sync).
int sweep(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
          const double* freqs, int nfreq, int form, int batch, int iters, double* x_out, double* corr_out,
          bool wait_out = true);
void release_sweep(bem_ctx* ctx);
void release_sweep_graph(bem_ctx* ctx);
// Lockstep solve of problems of uneven size (bem_batch_solve).
int batch_solve(bem_ctx* driver, int nprob, bem_ctx* const* probs, const double* freqs, const double* zge,
                const double* zcs, const double* zcp, const double* c, int form, int iters, double* const* x_out,
                double* corr_out);
// Serving (one problem per context): bytes a cached problem of size nn keeps
// on the device; enqueue a full solve (assembly + LU (+ refinement), keeping
// the post-swap G) or a right-hand-side-only solve with the cached factors,
// asynchronously on ctx->stream; the raw solution's device address.
size_t slot_footprint(int nn, int nbe, int ng, bool mixed);
int slot_solve_full(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                    double fr, bool mixed, int iters);
int slot_solve_rhs(bem_ctx* ctx, bool mixed, int iters);
const double2* slot_solution(bem_ctx* ctx, bool mixed, bool rhs_only);
// `batch` frequencies with the same boundary conditions in one lockstep step
// (not cached for right-hand-side reuse); problem b's raw solution.
int slot_solve_batch(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], const double c[4],
                     const double* freqs, int batch, bool mixed, int iters);
const double2* slot_batch_solution(bem_ctx* ctx, bool mixed, int b);

// Tensor-core FP32 trailing update (gemm_tc.cu).
int tc_ensure(bem_ctx* ctx, int nn, int batch);
void tc_release(bem_ctx* ctx);
int tc_trailing_update(bem_ctx* ctx, float2* A, size_t lda, size_t bstride, int nn, int k, int w, int batch);
int tc_pack_l(bem_ctx* ctx, const float2* A, size_t lda, size_t bstride, int nn, int kcol, int kw, int r0, int koff,
              int batch, const int* gmap, size_t gstride, int npanels = 1, int nmaps = 1);
int tc_gemm(bem_ctx* ctx, float2* A, size_t lda, size_t bstride, int nn, int r0, int c0, int cend, int kw,
            int urow_off, int batch, int kbase);
constexpr int kTcKPitch = 256;  // floats per packed tensor-core operand row

// One 32-row block of the packed tensor-core operand Lhat (256 threads):
// L(r, k..k+kw-1) for rows rbase..rbase+31 (L's storage row map[r], or r)
// goes to rows 2(r - r0) + part of `out`, K slots koff..koff+kw-1, rounded to
// TF32.  Uses a [64][33] shared tile and 32 shared ints; the caller
// synchronises before the next block reuses them.
__device__ __forceinline__ void pack_l_rows(const float2* __restrict__ Ap, size_t lda, int nn, int k, int kw, int r0,
                                            int rbase, int koff, float* out, const int* __restrict__ map,
                                            float2 (*tile)[33], int* s_src) {
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 x 32
  if (threadIdx.x < 32) {
    const int r = rbase + threadIdx.x;
    s_src[threadIdx.x] = (map && r < nn) ? map[r] : r;
  }
  __syncthreads();
  const int src = s_src[tx];
  for (int c = ty; c < 64; c += 8) {
    const int r = rbase + tx;
    float2 v = make_float2(0.f, 0.f);
    if (c < kw && r < nn) v = Ap[(size_t)(k + c) * lda + src];
    tile[c][tx] = v;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 32 * 2 * 64; idx += blockDim.x) {
    const int c = idx & 63, rr = idx >> 6;  // rr = 2*local_row + part
    const int lr = rr >> 1, part = rr & 1;
    const int r = rbase + lr;
    if (r >= nn || c >= kw) continue;
    const float2 v = tile[c][lr];
    unsigned t;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t) : "f"(part ? v.y : v.x));
    out[(size_t)(2 * (r - r0) + part) * kTcKPitch + koff + c] = __uint_as_float(t);
  }
}
int measure_fp64_peak(bem_ctx* ctx, double* tflops);
int measure_fma_peaks(bem_ctx* ctx, double* fp64_tflops, double* fp32_tflops);
int measure_tf32_peak(bem_ctx* ctx, int n, double* tflops);

int check_status(bem_ctx* ctx);
// The failure-path self-test kernel (bem_wait_selftest), lu.cu.
int wait_selftest(bem_ctx* ctx, int which);

}  // namespace bem
