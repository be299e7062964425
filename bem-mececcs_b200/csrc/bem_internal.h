// bem_internal.h -- the context behind the C-ABI and the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "bem_capi.h"
#include "bem_device.cuh"

namespace bem {

// Largest Gauss rule per direction (the reference's fixtures use 8).
constexpr int kMaxNpg = 8;

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

struct LuWork {
  int cap_nn = 0;
  int* ipiv = nullptr;          // [nn] 1-based pivot rows
  int* perm = nullptr;          // [2 + 4*64] count, then dst/src pairs of one panel
  double* slot_val = nullptr;   // [2][kMaxGrid]
  int* slot_row = nullptr;      // [2][kMaxGrid]
  double2* cand = nullptr;      // [2][kMaxGrid][64]
  double2* drow = nullptr;      // [2][64]
  unsigned* barrier = nullptr;  // grid barrier counter
};

constexpr int kMaxGrid = 160;

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
};

// Brackets one launch of class `cls` with events when profiling is on.
struct ProfScope {
  bem_ctx* ctx;
  int cls;
  cudaEvent_t b = nullptr;
  ProfScope(bem_ctx* c, int k, double work);
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
};

namespace bem {

int fail(bem_ctx* ctx, int code, const std::string& msg);
int cuda_fail(bem_ctx* ctx, cudaError_t e, const char* what);

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

// LU (lu.cu).
int lu_ensure_workspace(bem_ctx* ctx, int nn);
int lu_factor_solve(bem_ctx* ctx);
int measure_fp64_peak(bem_ctx* ctx, double* tflops);

int check_status(bem_ctx* ctx);

}  // namespace bem
