// lu.cu -- dense complex LU with partial pivoting and solve (FP64 form).
//
// Replaces LINSOLVE's ZGESV (src/Linsolve.for:94-100) and the reference's
// magma_zgesv_gpu (src/kernels/Linsolve_cu.cu:86-89).  Blocked right-looking
// factorisation of A = [ZH | ZFI] (the right-hand side rides along as column
// nn, so the forward substitution happens during the factorisation):
//
//   for each panel of NB columns starting at k:
//     k_panel        cooperative kernel; the panel's rows live in shared
//                    memory spread over up to one CTA per SM; one bounded
//                    grid barrier per column; pivot = first row of largest
//                    |re|+|im| (LAPACK IZAMAX), rows interchanged as ZGETF2.
//     k_laswp_trsm   the panel's row interchanges applied to every column
//                    to the right (as one gather) and U12 = L11^-1 A12.
//     k_gemm_update  A22 -= L21 U12 on the FP64 tensor cores (DMMA
//                    m8n8k4), complex as 4 real products.
//   k_backsub        U x = y, one launch per NB-row block.
//
// Row interchanges are never applied to the columns left of a panel: the
// solve does not need L in LAPACK's final row order.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "bem_internal.h"

namespace bem {

constexpr int kPanelThreads = 256;
constexpr int kPermMax = 2 * 64;  // perm list capacity of one panel

struct PanelArgs {
  double2* A;
  size_t lda;
  int nn, k, w, G, R;
  int* ipiv;
  int* perm;
  double* slot_val;
  int* slot_row;
  double2* cand;
  double2* drow;
  unsigned* bar;
  int* status;
};

__device__ __forceinline__ zd ldz(const double2* p) {
  double2 v = *p;
  return zd{v.x, v.y};
}
__device__ __forceinline__ zd ldz_cg(const double2* p) {
  double2 v = __ldcg(p);
  return zd{v.x, v.y};
}
__device__ __forceinline__ void stz(double2* p, zd z) { *p = make_double2(z.re, z.im); }

__device__ __forceinline__ bool better(double v, int r, double bv, int br) {
  return v > bv || (v == bv && r < br);
}

template <int NB>
__global__ void __launch_bounds__(kPanelThreads) k_panel(PanelArgs a) {
  extern __shared__ __align__(16) double2 s_raw[];
  zd* s_a = reinterpret_cast<zd*>(s_raw);  // [NB][R], column-major panel rows
  __shared__ zd s_piv[NB], s_drow[NB];
  __shared__ double s_rv[kPanelThreads / 32];
  __shared__ int s_rr[kPanelThreads / 32];
  __shared__ int s_best, s_win_row, s_win_cta;
  __shared__ int s_pdst[kPermMax], s_psrc[kPermMax];
  __shared__ int s_pcount;

  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int R = a.R, w = a.w, k = a.k;
  const int rbase = k + b * R;
  const int rcount = max(0, min(R, a.nn - rbase));

  for (int idx = tid; idx < w * rcount; idx += blockDim.x) {
    const int c = idx / rcount, r = idx % rcount;
    s_a[c * R + r] = ldz(&a.A[(size_t)(k + c) * a.lda + rbase + r]);
  }
  if (b == 0 && tid < w) {
    s_pdst[tid] = k + tid;
    s_psrc[tid] = k + tid;
  }
  if (b == 0 && tid == 0) s_pcount = w;
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int gj = k + j;
    const int par = j & 1;
    // 1. Local candidate: first row of largest |re|+|im| in column j.
    double bv = -1.0;
    int br = INT_MAX;
    for (int r = tid; r < rcount; r += blockDim.x) {
      const int gr = rbase + r;
      if (gr >= gj) {
        const double v = cabs1(s_a[j * R + r]);
        if (better(v, gr, bv, br)) {
          bv = v;
          br = gr;
        }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int orr = __shfl_xor_sync(0xffffffffu, br, off);
      if (better(ov, orr, bv, br)) {
        bv = ov;
        br = orr;
      }
    }
    if (lane == 0) {
      s_rv[warp] = bv;
      s_rr[warp] = br;
    }
    __syncthreads();
    if (tid == 0) {
      double v = s_rv[0];
      int rr = s_rr[0];
      for (int q = 1; q < kPanelThreads / 32; ++q)
        if (better(s_rv[q], s_rr[q], v, rr)) {
          v = s_rv[q];
          rr = s_rr[q];
        }
      a.slot_val[par * a.G + b] = v;
      a.slot_row[par * a.G + b] = rr;
      s_best = rr;
    }
    __syncthreads();
    // 2. Publish the candidate row and, from its owner, the current row gj.
    const int lbr = s_best;
    if (lbr != INT_MAX && tid < w)
      stz(&a.cand[((size_t)par * a.G + b) * NB + tid], s_a[tid * R + (lbr - rbase)]);
    if (gj >= rbase && gj < rbase + rcount && tid < w)
      stz(&a.drow[par * NB + tid], s_a[tid * R + (gj - rbase)]);
    // 3. Everyone's candidates are visible after the barrier.
    if (!grid_barrier(a.bar, (unsigned)(j + 1), (unsigned)a.G, a.status)) return;
    if (tid == 0) __threadfence();
    if (warp == 0) {
      double v = -1.0;
      int rr = INT_MAX, cb = 0;
      for (int t = lane; t < a.G; t += 32) {
        const double tv = __ldcg(&a.slot_val[par * a.G + t]);
        const int tr = __ldcg(&a.slot_row[par * a.G + t]);
        if (better(tv, tr, v, rr)) {
          v = tv;
          rr = tr;
          cb = t;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int orr = __shfl_xor_sync(0xffffffffu, rr, off);
        const int ocb = __shfl_xor_sync(0xffffffffu, cb, off);
        if (better(ov, orr, v, rr)) {
          v = ov;
          rr = orr;
          cb = ocb;
        }
      }
      if (lane == 0) {
        s_win_row = rr;
        s_win_cta = cb;
      }
    }
    __syncthreads();
    const int prow = s_win_row, pcta = s_win_cta;
    if (tid < w) {
      s_piv[tid] = ldz_cg(&a.cand[((size_t)par * a.G + pcta) * NB + tid]);
      s_drow[tid] = ldz_cg(&a.drow[par * NB + tid]);
    }
    __syncthreads();
    // 4. Interchange rows gj and prow (ZGETF2 swaps whole panel rows).
    if (prow != gj && prow >= rbase && prow < rbase + rcount && tid < w)
      s_a[tid * R + (prow - rbase)] = s_drow[tid];
    if (gj >= rbase && gj < rbase + rcount && tid < w) s_a[tid * R + (gj - rbase)] = s_piv[tid];
    if (b == 0 && tid == 0) {
      a.ipiv[gj] = prow + 1;
      int ip;
      if (prow < k + w) {
        ip = prow - k;
      } else {
        ip = -1;
        for (int e = w; e < s_pcount; ++e)
          if (s_pdst[e] == prow) {
            ip = e;
            break;
          }
        if (ip < 0) {
          ip = s_pcount++;
          s_pdst[ip] = prow;
          s_psrc[ip] = prow;
        }
      }
      const int t = s_psrc[j];
      s_psrc[j] = s_psrc[ip];
      s_psrc[ip] = t;
    }
    __syncthreads();
    // 5. Multipliers L(:,j) = A(:,j) / pivot, then the rank-1 update of the
    //    panel columns right of j.  A zero pivot leaves the column as is and
    //    records the first such column (ZGETF2's INFO).
    const zd pv = s_piv[j];
    const bool zero = (pv.re == 0.0 && pv.im == 0.0);
    if (zero && b == 0 && tid == 0) atomicCAS(&a.status[ST_SINGULAR], 0, gj + 1);
    const zd rp = zero ? zd{0.0, 0.0} : crcp(pv);
    for (int r = tid; r < rcount; r += blockDim.x)
      if (rbase + r > gj) s_a[j * R + r] = s_a[j * R + r] * rp;
    __syncthreads();
    const int ncol = w - j - 1;
    for (int idx = tid; idx < ncol * rcount; idx += blockDim.x) {
      const int c = j + 1 + idx / rcount, r = idx % rcount;
      if (rbase + r > gj) {
        zd v = s_a[c * R + r];
        const zd l = s_a[j * R + r], u = s_piv[c];
        v.re = fma(-l.re, u.re, fma(l.im, u.im, v.re));
        v.im = fma(-l.re, u.im, fma(-l.im, u.re, v.im));
        s_a[c * R + r] = v;
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < w * rcount; idx += blockDim.x) {
    const int c = idx / rcount, r = idx % rcount;
    stz(&a.A[(size_t)(k + c) * a.lda + rbase + r], s_a[c * R + r]);
  }
  if (b == 0) {
    if (tid == 0) a.perm[0] = s_pcount;
    for (int e = tid; e < s_pcount; e += blockDim.x) {
      a.perm[1 + 2 * e] = s_pdst[e];
      a.perm[2 + 2 * e] = s_psrc[e];
    }
  }
}

// Row interchanges of one panel applied to columns [c0, ncols) as a gather,
// then U12 = L11^-1 A12 (unit lower).  One warp per column.
template <int NB>
__global__ void __launch_bounds__(256) k_laswp_trsm(double2* A, size_t lda, int k, int w, int c0, int ncols,
                                                    const int* __restrict__ perm) {
  extern __shared__ __align__(16) double2 s_raw[];
  zd* s_L = reinterpret_cast<zd*>(s_raw);  // [NB][NB] column-major
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    s_L[c * NB + r] = ldz(&A[(size_t)(k + c) * lda + k + r]);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int count = perm[0];
  const int* pl = perm + 1;
  constexpr int V = NB / 32;
  for (int col = c0 + blockIdx.x * 8 + warp; col < ncols; col += gridDim.x * 8) {
    double2* cp = A + (size_t)col * lda;
    zd v[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int e = lane + 32 * q;
      v[q] = (e < w) ? ldz(&cp[pl[2 * e + 1]]) : zd{0.0, 0.0};
    }
    zd x[2];
    int xd[2] = {-1, -1};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int e = w + lane + 32 * q;
      if (e < count) {
        xd[q] = pl[2 * e];
        x[q] = ldz(&cp[pl[2 * e + 1]]);
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q)
      if (xd[q] >= 0) stz(&cp[xd[q]], x[q]);
    // Forward substitution with the unit lower L11.
    for (int i = 0; i < w; ++i) {
      const int src = i & 31;
      zd ui;
#pragma unroll
      for (int q = 0; q < V; ++q)
        if ((i >> 5) == q) {
          ui.re = __shfl_sync(0xffffffffu, v[q].re, src);
          ui.im = __shfl_sync(0xffffffffu, v[q].im, src);
        }
#pragma unroll
      for (int q = 0; q < V; ++q) {
        const int r = lane + 32 * q;
        if (r > i && r < w) {
          const zd l = s_L[i * NB + r];
          v[q].re = fma(-l.re, ui.re, fma(l.im, ui.im, v[q].re));
          v[q].im = fma(-l.re, ui.im, fma(-l.im, ui.re, v[q].im));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int r = lane + 32 * q;
      if (r < w) stz(&cp[k + r], v[q]);
    }
  }
}

// ---------------------------------------------------------------------------
// Trailing update C -= A B on the FP64 tensor cores.
// C: rows [r0, nn), cols [c0, ncols); A = L21 (cols k..k+w); B = U12.
// CTA tile 64x64 complex, 8 warps of 32x16, k chunks of 16 double-buffered
// through cp.async.  Shared layouts keep every fragment load conflict-free:
// As[k][m] with row stride 66 and Bs[n][k] with stride 20 (complex units).
// ---------------------------------------------------------------------------
constexpr int GBM = 64, GBN = 64, GBK = 16;
constexpr int AS_STRIDE = GBM + 2;  // == 2 mod 8
constexpr int BS_STRIDE = GBK + 4;  // == 4 mod 8
constexpr size_t kGemmSmem = (size_t)2 * (GBK * AS_STRIDE + GBN * BS_STRIDE) * sizeof(double2);

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = smem_u32(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256) k_gemm_update(double2* A, size_t lda, int nn, int k, int w, int r0,
                                                     int c0, int ncols) {
  extern __shared__ __align__(16) double2 g_smem[];
  auto As = reinterpret_cast<double2(*)[GBK][AS_STRIDE]>(g_smem);
  auto Bs = reinterpret_cast<double2(*)[GBN][BS_STRIDE]>(g_smem + 2 * GBK * AS_STRIDE);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps
  const int row0 = r0 + blockIdx.x * GBM, col0 = c0 + blockIdx.y * GBN;

  auto load_chunk = [&](int stage, int kc) {
    // A tile: 16 k x 64 rows = 1024 complex, 4 per thread.
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int kk = idx >> 6, m = idx & 63;
      const int gr = row0 + m, gk = kc + kk;
      const bool ok = gr < nn && gk < w;
      const double2* src = ok ? &A[(size_t)(k + gk) * lda + gr] : A;
      cp_async16(&As[stage][kk][m], src, ok);
    }
    // B tile: 64 cols x 16 k = 1024 complex.
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int n = idx >> 4, kk = idx & 15;
      const int gc = col0 + n, gk = kc + kk;
      const bool ok = gc < ncols && gk < w;
      const double2* src = ok ? &A[(size_t)gc * lda + k + gk] : A;
      cp_async16(&Bs[stage][n][kk], src, ok);
    }
    cp_async_commit();
  };

  double acc_re[4][2][2], acc_im[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc_re[i][j][0] = acc_re[i][j][1] = acc_im[i][j][0] = acc_im[i][j][1] = 0.0;

  const int nchunks = (w + GBK - 1) / GBK;
  load_chunk(0, 0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk((c + 1) & 1, (c + 1) * GBK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int st = c & 1;
#pragma unroll
    for (int ks = 0; ks < GBK / 4; ++ks) {
      double2 af[4], bf[2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) af[mt] = As[st][ks * 4 + t][wm * 32 + mt * 8 + g];
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) bf[nt] = Bs[st][wn * 16 + nt * 8 + g][ks * 4 + t];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          dmma(acc_re[mt][nt][0], acc_re[mt][nt][1], af[mt].x, bf[nt].x);
          dmma(acc_re[mt][nt][0], acc_re[mt][nt][1], -af[mt].y, bf[nt].y);
          dmma(acc_im[mt][nt][0], acc_im[mt][nt][1], af[mt].x, bf[nt].y);
          dmma(acc_im[mt][nt][0], acc_im[mt][nt][1], af[mt].y, bf[nt].x);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int gr = row0 + wm * 32 + mt * 8 + g;
        const int gc = col0 + wn * 16 + nt * 8 + 2 * t + e;
        if (gr < nn && gc < ncols) {
          double2* p = &A[(size_t)gc * lda + gr];
          double2 v = *p;
          v.x -= acc_re[mt][nt][e];
          v.y -= acc_im[mt][nt][e];
          *p = v;
        }
      }
}

// ---------------------------------------------------------------------------
// Back substitution U x = y (y = column nn of A after the factorisation).
// Launch s handles block s (rows [s*NB, ...)): every row above block s+1
// first subtracts U(row, block s+1) x_{s+1}; CTA 0 owns the rows of block s
// and then solves its upper-triangular diagonal block.
// ---------------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(256) k_backsub(double2* A, size_t lda, int nn, int s) {
  __shared__ zd s_x[NB];
  __shared__ zd s_y[NB];
  double2* y = A + (size_t)nn * lda;
  const int b0 = s * NB, b1 = min(b0 + NB, nn);   // block s
  const int n0 = b1, n1 = min(b1 + NB, nn);       // block s+1 (already solved)
  const int wn = n1 - n0;
  for (int i = threadIdx.x; i < wn; i += blockDim.x) s_x[i] = ldz(&y[n0 + i]);
  __syncthreads();
  // Rows handled by this CTA.
  int lo, hi;
  if (blockIdx.x == 0) {
    lo = b0;
    hi = b1;
  } else {
    lo = (blockIdx.x - 1) * blockDim.x;
    hi = min(lo + (int)blockDim.x, b0);
  }
  const int r = lo + threadIdx.x;
  zd acc{0.0, 0.0};
  if (r < hi) {
    acc = ldz(&y[r]);
    for (int c = 0; c < wn; ++c) {
      const zd u = ldz(&A[(size_t)(n0 + c) * lda + r]);
      const zd xc = s_x[c];
      acc.re = fma(-u.re, xc.re, fma(u.im, xc.im, acc.re));
      acc.im = fma(-u.re, xc.im, fma(-u.im, xc.re, acc.im));
    }
    if (blockIdx.x != 0) stz(&y[r], acc);
  }
  if (blockIdx.x != 0) return;
  if (r < hi) s_y[r - b0] = acc;
  __syncthreads();
  // Upper-triangular solve of block s by warp 0 (2 rows per lane for NB=64).
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const int wb = b1 - b0;
  constexpr int V = NB / 32;
  zd v[V];
#pragma unroll
  for (int q = 0; q < V; ++q) {
    const int rr = lane + 32 * q;
    v[q] = rr < wb ? s_y[rr] : zd{0.0, 0.0};
  }
  for (int i = wb - 1; i >= 0; --i) {
    const int srcl = i & 31;
    zd yi;
#pragma unroll
    for (int q = 0; q < V; ++q)
      if ((i >> 5) == q) {
        yi.re = __shfl_sync(0xffffffffu, v[q].re, srcl);
        yi.im = __shfl_sync(0xffffffffu, v[q].im, srcl);
      }
    const zd d = ldz(&A[(size_t)(b0 + i) * lda + b0 + i]);
    // x_i = y_i / U_ii
    const double den = 1.0 / fma(d.re, d.re, d.im * d.im);
    const zd xi{(yi.re * d.re + yi.im * d.im) * den, (yi.im * d.re - yi.re * d.im) * den};
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int rr = lane + 32 * q;
      if (rr == i) v[q] = xi;
      if (rr < i) {
        const zd u = ldz(&A[(size_t)(b0 + i) * lda + b0 + rr]);
        v[q].re = fma(-u.re, xi.re, fma(u.im, xi.im, v[q].re));
        v[q].im = fma(-u.re, xi.im, fma(-u.im, xi.re, v[q].im));
      }
    }
  }
#pragma unroll
  for (int q = 0; q < V; ++q) {
    const int rr = lane + 32 * q;
    if (rr < wb) stz(&y[b0 + rr], v[q]);
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
int lu_ensure_workspace(bem_ctx* ctx, int nn) {
  LuWork& L = ctx->lu;
  if (L.cap_nn >= nn && L.ipiv) return BEM_OK;
  cudaFree(L.ipiv);
  L.ipiv = nullptr;
  BEM_CUDA(ctx, cudaMalloc(&L.ipiv, (size_t)nn * sizeof(int)));
  L.cap_nn = nn;
  if (!L.perm) {
    BEM_CUDA(ctx, cudaMalloc(&L.perm, (1 + 2 * kPermMax) * sizeof(int)));
    BEM_CUDA(ctx, cudaMalloc(&L.slot_val, 2 * kMaxGrid * sizeof(double)));
    BEM_CUDA(ctx, cudaMalloc(&L.slot_row, 2 * kMaxGrid * sizeof(int)));
    BEM_CUDA(ctx, cudaMalloc(&L.cand, (size_t)2 * kMaxGrid * 64 * sizeof(double2)));
    BEM_CUDA(ctx, cudaMalloc(&L.drow, 2 * 64 * sizeof(double2)));
    BEM_CUDA(ctx, cudaMalloc(&L.barrier, sizeof(unsigned)));
  }
  return BEM_OK;
}

template <int NB>
static int lu_run(bem_ctx* ctx) {
  System& s = ctx->sys;
  LuWork& L = ctx->lu;
  const int nn = s.nn;
  const int ncols = nn + 1;
  {
    BEM_CUDA(ctx, cudaFuncSetAttribute(k_panel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    BEM_CUDA(ctx, cudaFuncSetAttribute(k_laswp_trsm<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       NB * NB * (int)sizeof(double2)));
    BEM_CUDA(ctx, cudaFuncSetAttribute(k_gemm_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kGemmSmem));
  }
  const int max_rows = (200 * 1024) / (NB * (int)sizeof(double2));
  for (int k = 0; k < nn; k += NB) {
    const int w = std::min(NB, nn - k);
    const int m = nn - k;
    int G = std::min({ctx->num_sms, kMaxGrid, (m + 15) / 16});
    G = std::max(G, 1);
    int R = (m + G - 1) / G;
    if (R > max_rows) return fail(ctx, BEM_ERR_ARG, "matrix too large for the FP64 panel kernel");
    G = (m + R - 1) / R;
    PanelArgs pa{s.A, s.lda, nn, k, w, G, R, L.ipiv, L.perm, L.slot_val, L.slot_row, L.cand, L.drow,
                 L.barrier, ctx->d_status};
    BEM_CUDA(ctx, cudaMemsetAsync(L.barrier, 0, sizeof(unsigned), ctx->stream));
    void* args[] = {&pa};
    const size_t smem = (size_t)R * NB * sizeof(double2);
    {
      ProfScope ps(ctx, 1, 0.0);
      BEM_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)k_panel<NB>, dim3(G), dim3(kPanelThreads), args,
                                                smem, ctx->stream));
    }
    ctx->launches++;
    const int c0 = k + w;
    if (c0 < ncols) {
      const int cols = ncols - c0;
      const int blocks = std::min((cols + 7) / 8, 4 * ctx->num_sms);
      {
        ProfScope ps(ctx, 2, 0.0);
        k_laswp_trsm<NB><<<blocks, 256, NB * NB * sizeof(double2), ctx->stream>>>(s.A, s.lda, k, w, c0, ncols,
                                                                                L.perm);
      }
      ctx->launches++;
      BEM_CUDA(ctx, cudaGetLastError());
      if (c0 < nn) {
        dim3 grid((nn - c0 + GBM - 1) / GBM, (cols + GBN - 1) / GBN);
        {
          ProfScope ps(ctx, 3, 8.0 * (double)(nn - c0) * (double)cols * (double)w);
          k_gemm_update<<<grid, 256, kGemmSmem, ctx->stream>>>(s.A, s.lda, nn, k, w, c0, c0, ncols);
        }
        ctx->launches++;
        BEM_CUDA(ctx, cudaGetLastError());
      }
    }
  }
  const int nblocks = (nn + NB - 1) / NB;
  ProfScope ps(ctx, 4, 0.0);
  for (int sblk = nblocks - 1; sblk >= 0; --sblk) {
    const int b0 = sblk * NB;
    const int grid = 1 + (b0 + 255) / 256;
    k_backsub<NB><<<grid, 256, 0, ctx->stream>>>(s.A, s.lda, nn, sblk);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
  }
  return BEM_OK;
}

// FP64 tensor-core throughput probe: independent DMMA chains in registers.
__global__ void __launch_bounds__(256) k_dmma_peak(double* out, int iters) {
  double acc[8][2];
#pragma unroll
  for (int q = 0; q < 8; ++q) acc[q][0] = acc[q][1] = 0.0;
  const double a = 1e-3 * (threadIdx.x + 1), b = 1e-3 * (blockIdx.x + 1);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) dmma(acc[q][0], acc[q][1], a, b);
  }
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) sum += acc[q][0] + acc[q][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = sum;
}

int measure_fp64_peak(bem_ctx* ctx, double* tflops) {
  const int blocks = ctx->num_sms * 4, threads = 256, iters = 8192;
  double* out = nullptr;
  cudaEvent_t e0, e1;
  BEM_CUDA(ctx, cudaMalloc(&out, (size_t)blocks * threads * sizeof(double)));
  BEM_CUDA(ctx, cudaEventCreate(&e0));
  BEM_CUDA(ctx, cudaEventCreate(&e1));
  k_dmma_peak<<<blocks, threads, 0, ctx->stream>>>(out, iters / 8);  // warm-up
  BEM_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  k_dmma_peak<<<blocks, threads, 0, ctx->stream>>>(out, iters);
  BEM_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
  ctx->launches += 2;
  BEM_CUDA(ctx, cudaEventSynchronize(e1));
  float ms = 0.f;
  BEM_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
  const double flops = (double)blocks * (threads / 32) * iters * 8 * 512.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return BEM_OK;
}

int lu_factor_solve(bem_ctx* ctx) {
  int rc = lu_ensure_workspace(ctx, ctx->sys.nn);
  if (rc) return rc;
  return lu_run<64>(ctx);
}

}  // namespace bem
