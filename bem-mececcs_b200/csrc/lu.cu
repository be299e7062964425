// lu.cu -- dense complex LU with partial pivoting and solve, FP64 and FP32.
//
// Replaces LINSOLVE's ZGESV (src/Linsolve.for:94-100) and the reference's
// magma_zgesv_gpu (src/kernels/Linsolve_cu.cu:86-89).  Blocked right-looking
// factorisation of A = [ZH | ZFI]: the right-hand side rides along as column
// nn, so the forward substitution happens during the factorisation.  A batch
// of B equal-size problems (A_b = A + b * bstride) is factored in lockstep.
//
//   for each panel of w columns starting at k (w adapts to the panel height):
//     k_panel_push     one thread-block cluster (16 CTAs) per problem holds the
//                      panel rows in shared memory; per column every CTA pushes
//                      its pivot candidate (and the owner row gj) into mailboxes
//                      in every CTA (st.async, counted by an mbarrier).  Pivot =
//                      first row of largest |re|+|im| (LAPACK IZAMAX); rows are
//                      interchanged as ZGETF2 does.  k_panel_cluster (pull form)
//                      and k_panel_calu (tournament pivoting) are options.
//     k_panel_grid     fallback for panels too tall for one cluster: the same
//                      algorithm over a cooperative grid with a bounded
//                      software grid barrier.
//     k_l11_inv +      FP32: L11^-1 once per panel, then the panel's row
//     k_laswp_tc       interchanges on every column to the right and U12 =
//                      L11^-1 A12 on TF32 tensor cores (with the deferred update
//                      of the earlier panels of a group); k_laswp_trsm does the
//                      same by substitution (FP64).
//     k_gemm_f64       A22 -= L21 U12 on the FP64 tensor cores (DMMA m8n8k4).
//     k_gemm_tc        (gemm_tc.cu) the FP32 update on tcgen05, K = 64 G for a
//                      group of G = 1, 2 or 4 panels; k_gemm_tf32 on mma.sync.
//   k_trsv_f32 /       forward + back substitution in one cooperative launch
//   k_trsv             (FP32 with inverted diagonal blocks from k_tri_inv;
//                      FP64 by substitution); k_backsub per 64-row block.
//
// Row interchanges are never applied to columns left of a panel; each panel's
// interchanges are kept (ipiv and a dst/src gather list) so that later solves
// can replay them in panel order.
#include <cublas_v2.h>
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "bem_internal.h"

namespace bem {

constexpr int kPanelThreads = 256;

template <typename R>
struct Elt;
template <>
struct Elt<double> {
  using T = double2;
};
template <>
struct Elt<float> {
  using T = float2;
};

template <typename R>
__device__ __forceinline__ cpx<R> ldc(const typename Elt<R>::T* p) {
  const auto v = *p;
  return cpx<R>{v.x, v.y};
}
template <typename R>
__device__ __forceinline__ cpx<R> ldc_cg(const typename Elt<R>::T* p) {
  const auto v = __ldcg(p);
  return cpx<R>{v.x, v.y};
}
template <typename R>
__device__ __forceinline__ void stc(typename Elt<R>::T* p, cpx<R> z) {
  typename Elt<R>::T v;
  v.x = z.re;
  v.y = z.im;
  *p = v;
}
// a -= l * u
template <typename R>
__device__ __forceinline__ void cfms(cpx<R>& a, cpx<R> l, cpx<R> u) {
  a.re = fma(-l.re, u.re, fma(l.im, u.im, a.re));
  a.im = fma(-l.re, u.im, fma(-l.im, u.re, a.im));
}

template <typename R>
__device__ __forceinline__ bool better(R v, int r, R bv, int br) {
  return v > bv || (v == bv && r < br);
}

// ---- thread-block cluster helpers (distributed shared memory) ----
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned map_rank(const void* p, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ int dsm_ld(const int* p, unsigned rank) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(map_rank(p, rank)) : "memory");
  return v;
}
__device__ __forceinline__ double dsm_ld(const double* p, unsigned rank) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(map_rank(p, rank)) : "memory");
  return v;
}
__device__ __forceinline__ float dsm_ld(const float* p, unsigned rank) {
  float v;
  asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(map_rank(p, rank)) : "memory");
  return v;
}
__device__ __forceinline__ zd dsm_ld(const zd* p, unsigned rank) {
  zd v;
  asm volatile("ld.shared::cluster.v2.f64 {%0,%1}, [%2];" : "=d"(v.re), "=d"(v.im) : "r"(map_rank(p, rank)) : "memory");
  return v;
}
__device__ __forceinline__ zf dsm_ld(const zf* p, unsigned rank) {
  zf v;
  asm volatile("ld.shared::cluster.v2.f32 {%0,%1}, [%2];" : "=f"(v.re), "=f"(v.im) : "r"(map_rank(p, rank)) : "memory");
  return v;
}

// Four consecutive complex values of a shared-memory row (16-byte aligned
// for float: two 16-byte broadcast loads instead of four 8-byte ones).
__device__ __forceinline__ void ld4(const zf* p, zf (&o)[4]) {
  const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
  o[0] = zf{a.x, a.y};
  o[1] = zf{a.z, a.w};
  o[2] = zf{b.x, b.y};
  o[3] = zf{b.z, b.w};
}
__device__ __forceinline__ void ld4(const zd* p, zd (&o)[4]) {
#pragma unroll
  for (int u = 0; u < 4; ++u) o[u] = p[u];
}

// Shared state of one problem's panel step.
struct PanelArgs {
  void* A;
  size_t lda, bstride;
  int nn, k, w;
  int rp;          // panel rows per CTA
  int cs;          // CTAs per problem (cluster size or grid size)
  int* ipiv;       // [B][nn] 1-based pivot rows
  int ipiv_stride;
  int* perm;       // [B][kPermStride]: count, then dst/src pairs
  int perm_stride;
  int* status;
  int* pstart;     // panel starts for the later solves: [pidx] = k, [pidx + 1] = k + w
  int pidx;
  int async_mail;  // k_panel_push: mailboxes filled by st.async (mbarrier complete_tx), no per-column cluster barrier
  int no_singular;  // a tournament round of a tall panel: a zero pivot is not an error here
  // grid fallback only:
  void* slot_val;
  int* slot_row;
  void* cand;
  void* drow;
  unsigned* bar;
};

// Per-column bookkeeping of the gather list that replays the panel's row
// interchanges on other columns: entries 0..w-1 are rows k..k+w-1, entries
// beyond w are displaced rows below the panel.  Called by one thread.
__device__ __forceinline__ void perm_swap(int* pdst, int* psrc, int& pcount, int k, int w, int j, int prow) {
  int ip;
  if (prow < k + w) {
    ip = prow - k;
  } else {
    ip = -1;
    for (int e = w; e < pcount; ++e)
      if (pdst[e] == prow) {
        ip = e;
        break;
      }
    if (ip < 0) {
      ip = pcount++;
      pdst[ip] = prow;
      psrc[ip] = prow;
    }
  }
  const int t = psrc[j];
  psrc[j] = psrc[ip];
  psrc[ip] = t;
}

// Local part of every column step: candidate search over the CTA's rows.
template <typename R>
__device__ __forceinline__ void local_argmax(const cpx<R>* col, int rcount, int rbase, int gj, R* s_rv, int* s_rr,
                                             R& out_v, int& out_r) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  R bv = R(-1);
  int br = INT_MAX;
  for (int r = tid; r < rcount; r += blockDim.x) {
    const int gr = rbase + r;
    if (gr >= gj) {
      const R v = cabs1(col[r]);
      if (better(v, gr, bv, br)) {
        bv = v;
        br = gr;
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const R ov = __shfl_xor_sync(0xffffffffu, bv, off);
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
  R v = s_rv[0];
  int rr = s_rr[0];
  for (int q = 1; q < kPanelThreads / 32; ++q)
    if (better(s_rv[q], s_rr[q], v, rr)) {
      v = s_rv[q];
      rr = s_rr[q];
    }
  out_v = v;
  out_r = rr;
}

// Scale column j and apply the rank-1 update to the panel columns right of j.
// Rows [row0, row0 + rcount) x columns [col0, col0 + w) of A into s
// (column-major, leading dimension rp) with one cp.async per element: every
// copy is in flight before the single wait, so the slice costs one memory
// round trip rather than one per loop iteration.
template <typename R>
__device__ __forceinline__ void load_slice_async(const typename Elt<R>::T* A, size_t lda, int row0, int col0,
                                                 int rcount, int w, cpx<R>* s, int rp) {
  constexpr int kBytes = (int)sizeof(typename Elt<R>::T);
  for (int r = threadIdx.x; r < rcount; r += blockDim.x)
    for (int c = 0; c < w; ++c) {
      const unsigned dst = smem_u32(&s[(size_t)c * rp + r]);
      const void* src = &A[(size_t)(col0 + c) * lda + row0 + r];
      if constexpr (kBytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
    }
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

template <typename R>
__device__ __forceinline__ void eliminate(cpx<R>* s_a, int rp, int rcount, int rbase, int gj, int j, int w,
                                          const cpx<R>* s_piv, int* status, bool report) {
  const int tid = threadIdx.x;
  const cpx<R> pv = s_piv[j];
  const bool zero = (pv.re == R(0) && pv.im == R(0));
  if (zero && report && tid == 0) atomicCAS(&status[ST_SINGULAR], 0, gj + 1);
  const cpx<R> rpv = zero ? cpx<R>{R(0), R(0)} : crcp(pv);
  for (int r = tid; r < rcount; r += blockDim.x)
    if (rbase + r > gj) s_a[j * rp + r] = s_a[j * rp + r] * rpv;
  __syncthreads();
  const int ncol = w - j - 1;
  for (int idx = tid; idx < ncol * rcount; idx += blockDim.x) {
    const int c = j + 1 + idx / rcount, r = idx % rcount;
    if (rbase + r > gj) cfms(s_a[c * rp + r], s_a[j * rp + r], s_piv[c]);
  }
  __syncthreads();
}

// Panel factorisation in one thread-block cluster per problem.  CTA `rank`
// owns panel rows [k + rank*rp, ...) in shared memory; thread t owns local
// rows t, t+256, ... (RPT of them).  The panel is processed in sub-panels of
// 8 columns held in registers, so the per-column rank-1 updates never touch
// shared memory; the columns right of a sub-panel are updated once per
// sub-panel (a triangular solve of the sub-panel's 8 pivot rows, then a
// rank-8 update).  Per column: one CTA barrier and one cluster barrier; the
// pivot candidates and the pivot row are read over distributed shared
// memory from double-buffered publish areas.
template <typename R, int NB, int NT>
__global__ void __launch_bounds__(NT, 1) k_panel_cluster(PanelArgs a) {
  constexpr int RPT = 1;
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  constexpr int SW = 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_a = reinterpret_cast<C*>(smem_raw);  // [NB][rp] panel rows, column-major
  C* s_pub = s_a + (size_t)NB * a.rp;       // [2][2][NB]: candidate row, row gj
  C* s_blk = s_pub + 4 * NB;                // [2][SW][NB]: a sub-panel's pivot rows
  __shared__ __align__(16) C s_u[SW][NB];   // U of the sub-panel's pivot rows (16-byte rows for ld4)
  __shared__ R s_pval[2];
  __shared__ int s_prow[2];
  __shared__ R s_rv[NT / 32];
  __shared__ int s_rr[NT / 32];
  __shared__ int s_pdst[2 * NB], s_psrc[2 * NB];
  __shared__ int s_pcount;
  __shared__ int s_ipiv[NB];
  __shared__ C s_pv[8];        // pivot row, sub-panel columns
  __shared__ int s_win[2];     // winner row, winner rank

  const unsigned rank = cluster_rank();
  const int prob = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  E* A = static_cast<E*>(a.A) + (size_t)prob * a.bstride;
  int* ipiv = a.ipiv + (size_t)prob * a.ipiv_stride;
  int* perm = a.perm + (size_t)prob * a.perm_stride;
  const int rp = a.rp, w = a.w, k = a.k, cs = a.cs;
  const int rbase = k + (int)rank * rp;
  const int rcount = max(0, min(rp, a.nn - rbase));

  load_slice_async<R>(A, a.lda, rbase, k, rcount, w, s_a, rp);
  if (rank == 0 && prob == 0 && tid == 0 && a.pstart) {
    a.pstart[a.pidx] = k;
    a.pstart[a.pidx + 1] = k + w;
  }
  if (rank == 0 && tid < w) {
    s_pdst[tid] = k + tid;
    s_psrc[tid] = k + tid;
  }
  if (rank == 0 && tid == 0) s_pcount = w;
  __syncthreads();

  // Global row of my q-th local row (INT_MAX when it does not exist).
  int grow[RPT];
#pragma unroll
  for (int q = 0; q < RPT; ++q) {
    const int lr = tid + NT * q;
    grow[q] = lr < rcount ? rbase + lr : INT_MAX;
  }
  C v[RPT][SW];

  for (int s0 = 0; s0 < w; s0 += SW) {
    const int sw = min(SW, w - s0);
#pragma unroll
    for (int q = 0; q < RPT; ++q)
#pragma unroll
      for (int c = 0; c < SW; ++c)
        v[q][c] = (grow[q] != INT_MAX && c < sw) ? s_a[(s0 + c) * rp + (grow[q] - rbase)] : C{R(0), R(0)};

    for (int jj = 0; jj < sw; ++jj) {
      const int j = s0 + jj, gj = k + j, par = j & 1;
      const int owner = j / rp;  // (gj - k) / rp
      // 1. Candidate over my rows, then over the CTA.
      R bv = R(-1);
      int br = INT_MAX;
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        if (grow[q] != INT_MAX && grow[q] >= gj) {
          C x = v[q][0];
#pragma unroll
          for (int c = 1; c < SW; ++c)
            if (c == jj) x = v[q][c];
          const R val = cabs1(x);
          if (better(val, grow[q], bv, br)) {
            bv = val;
            br = grow[q];
          }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const R ov = __shfl_xor_sync(0xffffffffu, bv, off);
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
      R cv = s_rv[0];
      int cr = s_rr[0];
#pragma unroll
      for (int q = 1; q < NT / 32; ++q)
        if (better(s_rv[q], s_rr[q], cv, cr)) {
          cv = s_rv[q];
          cr = s_rr[q];
        }
      // 2. Publish the candidate row and, from its owner, row gj.
      C* cand = s_pub + (size_t)par * 2 * NB;
      C* drow = cand + NB;
      if (tid == 0) {
        s_pval[par] = cv;
        s_prow[par] = cr;
      }
      if (cr != INT_MAX) {
        const int lr = cr - rbase;
        if (tid < w && (tid < s0 || tid >= s0 + sw)) cand[tid] = s_a[tid * rp + lr];
        if (tid == (lr & (NT - 1))) {
#pragma unroll
          for (int q = 0; q < RPT; ++q)
            if (q == (lr / NT))
#pragma unroll
              for (int c = 0; c < SW; ++c)
                if (c < sw) cand[s0 + c] = v[q][c];
        }
      }
      if ((int)rank == owner) {
        const int lr = gj - rbase;
        if (tid < w && (tid < s0 || tid >= s0 + sw)) drow[tid] = s_a[tid * rp + lr];
        if (tid == (lr & (NT - 1))) {
#pragma unroll
          for (int q = 0; q < RPT; ++q)
            if (q == (lr / NT))
#pragma unroll
              for (int c = 0; c < SW; ++c)
                if (c < sw) drow[s0 + c] = v[q][c];
        }
      }
      cluster_sync();
      // 3. Winner: warp 0 reads every CTA's candidate (value, row and its 8
      //    sub-panel values) in one round of remote loads, reduces, and
      //    broadcasts through shared memory.
      if (warp == 0) {
        R wv = R(-1);
        int wr = INT_MAX, wk = 0;
        C cvals[SW];
#pragma unroll
        for (int c = 0; c < SW; ++c) cvals[c] = C{R(0), R(0)};
        if (lane < cs) {
          wv = dsm_ld(&s_pval[par], lane);
          wr = dsm_ld(&s_prow[par], lane);
          wk = lane;
#pragma unroll
          for (int c = 0; c < SW; ++c)
            if (c < sw) cvals[c] = dsm_ld(&cand[s0 + c], lane);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const R ov = __shfl_xor_sync(0xffffffffu, wv, off);
          const int orr = __shfl_xor_sync(0xffffffffu, wr, off);
          const int ok = __shfl_xor_sync(0xffffffffu, wk, off);
          if (better(ov, orr, wv, wr)) {
            wv = ov;
            wr = orr;
            wk = ok;
          }
        }
        // Lane wk holds the winner's values.
#pragma unroll
        for (int c = 0; c < SW; ++c) {
          const R re = __shfl_sync(0xffffffffu, cvals[c].re, wk);
          const R im = __shfl_sync(0xffffffffu, cvals[c].im, wk);
          if (lane == c) s_pv[c] = C{re, im};
        }
        if (lane == 0) {
          s_win[0] = wr;
          s_win[1] = wk;
        }
      }
      __syncthreads();
      const int prow = s_win[0];
      const unsigned wrank = (unsigned)s_win[1];
      C piv[SW];
#pragma unroll
      for (int c = 0; c < SW; ++c) piv[c] = s_pv[c];
      // 4. Interchange rows gj and prow (whole panel rows).
      if ((int)rank == owner && prow != gj) {  // row gj <- pivot row
        const int lr = gj - rbase;
        if (tid < w && (tid < s0 || tid >= s0 + sw)) s_a[tid * rp + lr] = dsm_ld(&cand[tid], wrank);
        if (tid == (lr & (NT - 1))) {
#pragma unroll
          for (int q = 0; q < RPT; ++q)
            if (q == (lr / NT))
#pragma unroll
              for (int c = 0; c < SW; ++c) v[q][c] = piv[c];
        }
      }
      if (prow != gj && prow >= rbase && prow < rbase + rcount) {  // row prow <- old row gj
        const int lr = prow - rbase;
        if (tid < w && (tid < s0 || tid >= s0 + sw)) s_a[tid * rp + lr] = dsm_ld(&drow[tid], (unsigned)owner);
        if (tid == (lr & (NT - 1))) {
#pragma unroll
          for (int q = 0; q < RPT; ++q)
            if (q == (lr / NT))
#pragma unroll
              for (int c = 0; c < SW; ++c)
                if (c < sw) v[q][c] = dsm_ld(&drow[s0 + c], (unsigned)owner);
        }
      }
      if (rank == 0 && tid == 0) {
        s_ipiv[j] = prow + 1;
        perm_swap(s_pdst, s_psrc, s_pcount, k, w, j, prow);
      }
      // 5. Multipliers and the rank-1 update of the sub-panel, in registers.
      C pj = piv[0];
#pragma unroll
      for (int c = 1; c < SW; ++c)
        if (c == jj) pj = piv[c];
      const bool zero = (pj.re == R(0) && pj.im == R(0));
      if (zero && rank == 0 && tid == 0 && !a.no_singular) atomicCAS(&a.status[ST_SINGULAR], 0, gj + 1);
      const C rpv = zero ? C{R(0), R(0)} : crcp(pj);
#pragma unroll
      for (int q = 0; q < RPT; ++q) {
        if (grow[q] != INT_MAX && grow[q] > gj) {
          C l = v[q][0];
#pragma unroll
          for (int c = 1; c < SW; ++c)
            if (c == jj) l = v[q][c];
          l = l * rpv;
#pragma unroll
          for (int c = 0; c < SW; ++c) {
            if (c == jj) v[q][c] = l;
            if (c > jj) cfms(v[q][c], l, piv[c]);
          }
        }
      }
    }
    // End of the sub-panel: registers back to shared memory.
#pragma unroll
    for (int q = 0; q < RPT; ++q)
      if (grow[q] != INT_MAX)
#pragma unroll
        for (int c = 0; c < SW; ++c)
          if (c < sw) s_a[(s0 + c) * rp + (grow[q] - rbase)] = v[q][c];
    if (s0 + sw >= w) break;
    // Publish this sub-panel's pivot rows (global rows k+s0 .. k+s0+sw-1).
    const int bpar = (s0 / SW) & 1;
    C* blk = s_blk + (size_t)bpar * SW * NB;
    __syncthreads();
    for (int idx = tid; idx < sw * w; idx += blockDim.x) {
      const int i = idx / w, c = idx % w;
      const int gr = k + s0 + i;
      if (gr >= rbase && gr < rbase + rcount) blk[i * NB + c] = s_a[c * rp + (gr - rbase)];
    }
    cluster_sync();
    for (int idx = tid; idx < sw * w; idx += blockDim.x) {
      const int i = idx / w, c = idx % w;
      s_u[i][c] = dsm_ld(&blk[i * NB + c], (unsigned)((s0 + i) / rp));
    }
    __syncthreads();
    // U of the pivot rows for the columns right of the sub-panel:
    // U(i,c) = A(i,c) - sum_{t<i} L(i,t) U(t,c), L = the sub-panel's unit lower.
    for (int c = s0 + sw + tid; c < w; c += blockDim.x)
      for (int i = 1; i < sw; ++i) {
        C x = s_u[i][c];
        for (int t = 0; t < i; ++t) cfms(x, s_u[i][s0 + t], s_u[t][c]);
        s_u[i][c] = x;
      }
    __syncthreads();
    // Rank-sw update of my rows in the columns right of the sub-panel; the
    // pivot rows themselves take their U values.
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int gr = grow[q];
      const int lr = gr - rbase;
      if (gr != INT_MAX && gr >= k + s0 + sw) {
        // Four columns per iteration as independent chains (the remaining
        // width is a multiple of 8).
        for (int c = s0 + sw; c < w; c += 4) {
          C x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) x[u] = s_a[(c + u) * rp + lr];
#pragma unroll
          for (int t = 0; t < SW; ++t)
            if (t < sw) {
              C uu[4];
              ld4(&s_u[t][c], uu);
#pragma unroll
              for (int u = 0; u < 4; ++u) cfms(x[u], v[q][t], uu[u]);
            }
#pragma unroll
          for (int u = 0; u < 4; ++u) s_a[(c + u) * rp + lr] = x[u];
        }
      } else if (gr != INT_MAX && gr >= k + s0) {
        const int i = gr - k - s0;
        for (int c = s0 + sw; c < w; ++c) s_a[c * rp + lr] = s_u[i][c];
      }
    }
    __syncthreads();
  }
  __syncthreads();
  for (int idx = tid; idx < w * rcount; idx += blockDim.x) {
    const int c = idx / rcount, r = idx % rcount;
    stc<R>(&A[(size_t)(k + c) * a.lda + rbase + r], s_a[c * rp + r]);
  }
  if (rank == 0) {
    if (tid < w) ipiv[k + tid] = s_ipiv[tid];
    if (tid == 0) perm[0] = s_pcount;
    for (int e = tid; e < s_pcount; e += blockDim.x) {
      perm[1 + 2 * e] = s_pdst[e];
      perm[2 + 2 * e] = s_psrc[e];
    }
  }
  cluster_sync();  // no CTA leaves while others may still read its shared memory
}

// ---------------------------------------------------------------------------
// Panel with tournament pivoting (FP32: the mixed form's factorisation, which
// only has to precondition the FP64 refinement).  Pivots are chosen per
// 8-column sub-panel instead of per column: every CTA picks 8 candidate rows
// of its own by partial pivoting on a copy of its rows (no cluster traffic),
// then every CTA gathers the cluster's candidates (cs x 8 rows) over
// distributed shared memory and runs the same partial pivoting on them, which
// yields the 8 pivot rows and the sub-panel's 8 x 8 L\U block in every CTA
// at once.  The 8 interchanges, applied in order as LAPACK would, move at
// most 16 rows; those rows are published and pulled in one more exchange, and
// every other row gets its L entries by a triangular solve against the U
// block.  Two cluster barriers per sub-panel instead of one per column.  The
// gather lists, pivot indices and the right-of-block update are those of
// k_panel_cluster, so the later kernels are unchanged.
// ---------------------------------------------------------------------------
constexpr int kCaluSW = 8;
constexpr int kCaluCand = 16 * kCaluSW;  // candidate rows of a 16-CTA cluster
constexpr int kCaluMoves = 2 * kCaluSW;  // rows that move (or pivot) per sub-panel

template <typename T, int N>
__device__ __forceinline__ T sel(const T (&x)[N], int j) {
  T r = x[0];
#pragma unroll
  for (int c = 1; c < N; ++c)
    if (c == j) r = x[c];
  return r;
}

// ---------------------------------------------------------------------------
// Panel factorisation in one thread-block cluster per problem, push form
// (the default).  Same partition as k_panel_cluster: CTA `rank` owns panel
// rows [k + rank*rp, ...) in shared memory, one row per thread, and the
// panel advances in 8-column sub-panels held in registers.  Every transfer
// of a column step is a remote STORE issued before the cluster barrier:
// each CTA pushes its candidate (|re| + |im|, row, and the row's 8 sub-panel
// values) into its mailbox slot in every CTA of the cluster, and the owner of
// row gj pushes that row's 8 sub-panel values the same way.  After the
// barrier every warp picks the winner from its own CTA's mailboxes, so a
// column costs one CTA barrier, one cluster barrier and no remote load.  The
// interchange acts at once on the sub-panel values in registers; the rest of
// the two rows (columns left and right of the sub-panel) moves once per
// sub-panel, as a list of row moves pulled over distributed shared memory
// after the sub-panel's own cluster barrier.  Pivot choice (LAPACK partial
// pivoting by |re| + |im|, first row on ties) and arithmetic are those of
// k_panel_cluster, so the factors are the same.
// ---------------------------------------------------------------------------
// TF32 tensor-core product of m16n8k8 fragments (FP32 accumulation); operands
// rounded to TF32 (round to nearest, ties away) first.
__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

constexpr int kPushMoves = 16;  // positions that a sub-panel's 8 interchanges can touch

// 16 bytes into CTA `rank`'s copy of p, completing that many bytes of the
// transaction count of its copy of mbarrier mb (the receiver waits on it).
__device__ __forceinline__ void dsm_st4_async(const void* p, unsigned rank, uint4 v, const uint64_t* mb) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(
                   map_rank(p, rank)),
               "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(map_rank(mb, rank))
               : "memory");
}
__device__ __forceinline__ void dsm_st4(const void* p, unsigned rank, uint4 v) {
  asm volatile("st.shared::cluster.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(map_rank(p, rank)), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w)
               : "memory");
}

// 8 sub-panel values of one row as 16-byte words (2 complex64 or 1 complex128
// per word), and a candidate's (value, row) word.
template <typename R>
struct RowWords {
  static constexpr int kN = sizeof(R) == 4 ? 4 : 8;
};
template <typename R>
__device__ __forceinline__ uint4 row_word(const cpx<R> (&x)[8], int q) {
  if constexpr (sizeof(R) == 4) {
    return make_uint4(__float_as_uint(x[2 * q].re), __float_as_uint(x[2 * q].im), __float_as_uint(x[2 * q + 1].re),
                      __float_as_uint(x[2 * q + 1].im));
  } else {
    const unsigned long long a = __double_as_longlong(x[q].re), b = __double_as_longlong(x[q].im);
    return make_uint4((unsigned)a, (unsigned)(a >> 32), (unsigned)b, (unsigned)(b >> 32));
  }
}
template <typename R>
__device__ __forceinline__ void row_unword(const uint4* wd, cpx<R> (&x)[8]) {
  if constexpr (sizeof(R) == 4) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 t = wd[q];
      x[2 * q] = cpx<R>{__uint_as_float(t.x), __uint_as_float(t.y)};
      x[2 * q + 1] = cpx<R>{__uint_as_float(t.z), __uint_as_float(t.w)};
    }
  } else {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const uint4 t = wd[q];
      x[q] = cpx<R>{__longlong_as_double((long long)(((unsigned long long)t.y << 32) | t.x)),
                    __longlong_as_double((long long)(((unsigned long long)t.w << 32) | t.z))};
    }
  }
}
template <typename R>
__device__ __forceinline__ uint4 cand_word(R v, int r) {
  if constexpr (sizeof(R) == 4) {
    return make_uint4(__float_as_uint(v), 0u, (unsigned)r, 0u);
  } else {
    const unsigned long long a = __double_as_longlong(v);
    return make_uint4((unsigned)a, (unsigned)(a >> 32), (unsigned)r, 0u);
  }
}
template <typename R>
__device__ __forceinline__ R cand_val(uint4 t) {
  if constexpr (sizeof(R) == 4)
    return __uint_as_float(t.x);
  else
    return __longlong_as_double((long long)(((unsigned long long)t.y << 32) | t.x));
}

template <typename R, int NB, int NT>
__global__ void __launch_bounds__(NT, 1) k_panel_push(PanelArgs a) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  constexpr int SW = 8, NW = NT / 32, KW = RowWords<R>::kN;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_a = reinterpret_cast<C*>(smem_raw);  // [NB][rp] panel rows, column-major
  C* s_pub = s_a + (size_t)NB * a.rp;       // [kPushMoves][NB] published rows (sub-panel start values)
  __shared__ uint4 s_box[2][16][1 + KW];    // [column parity][CTA]: candidate word, then its 8 values
  __shared__ uint4 s_dbox[2][KW];           // [column parity]: row gj's 8 values
  __shared__ uint4 s_wt[2][NW][KW];         // staged best row of every warp
  __shared__ uint4 s_gw[2][KW];             // staged row gj (its owner CTA)
  __shared__ __align__(16) C s_u[SW][NB];   // the sub-panel's pivot rows: L\U in the sub-panel, then U
  __shared__ R s_rv[2][NW];                 // per-warp candidates: value (FP64) or key (FP32), row
  __shared__ unsigned s_rk[2][NW];
  __shared__ int s_rr[2][NW];
  __shared__ int s_mdst[kPushMoves], s_msrc[kPushMoves], s_ment[kPushMoves], s_mcnt;
  const unsigned long long wlim = wait_limit(a.status);  // the context's bound on every wait
  __shared__ int s_ppos[kPushMoves], s_pcnt;  // published rows (positions)
  __shared__ int s_pent[SW];                  // published row holding each pivot row's right part
  __shared__ int s_pdst[2 * NB], s_psrc[2 * NB];
  __shared__ int s_pcount;
  __shared__ int s_ipiv[NB];
  __shared__ uint64_t s_mb[2];  // [column parity]: the mailboxes' arrivals (async_mail)

  const unsigned rank = cluster_rank();
  const int prob = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  E* A = static_cast<E*>(a.A) + (size_t)prob * a.bstride;
  int* ipiv = a.ipiv + (size_t)prob * a.ipiv_stride;
  int* perm = a.perm + (size_t)prob * a.perm_stride;
  const int rp = a.rp, w = a.w, k = a.k, cs = a.cs;
  const int rbase = k + (int)rank * rp;
  const int rcount = max(0, min(rp, a.nn - rbase));

  load_slice_async<R>(A, a.lda, rbase, k, rcount, w, s_a, rp);
  if (rank == 0 && prob == 0 && tid == 0 && a.pstart) {
    a.pstart[a.pidx] = k;
    a.pstart[a.pidx + 1] = k + w;
  }
  if (rank == 0 && tid < w) {
    s_pdst[tid] = k + tid;
    s_psrc[tid] = k + tid;
  }
  if (rank == 0 && tid == 0) s_pcount = w;
  const bool amail = a.async_mail != 0;
  if (amail && tid == 0) {
    mbar_init(&s_mb[0], 1);
    mbar_init(&s_mb[1], 1);
  }
  __syncthreads();
  if (amail) cluster_sync();  // every CTA's mbarriers exist before the first push
  // bytes arriving in a CTA per column: every CTA's candidate (1 + KW words) and row gj (KW words)
  const unsigned mail_bytes = (unsigned)(cs * (1 + KW) + KW) * 16u;
  unsigned mph = 0;  // phase bits of s_mb[0], s_mb[1]
  bool gave_up = false;  // this thread's mailbox wait ran out: later waits are skipped

  const int grow = tid < rcount ? rbase + tid : INT_MAX;  // my row (position)
  const C czero{R(0), R(0)};
  C v[SW];
  int swp[SW];  // pivot position chosen for each column of the sub-panel
  // Rank-sw update of my row over columns [c0, c1) by the sub-panel whose
  // pivot rows start at position ug0 (L of my row in lv, U in s_u); the
  // pivot rows themselves take their U values.  Column groups of 4 (a group
  // may run past w, into columns that are never stored).
  auto rank_update = [&](const C(&lv)[SW], int ug0, int usw, int c0, int c1) {
    if (grow == INT_MAX || grow < ug0) return;
    if (grow >= ug0 + usw) {
      for (int c = c0; c < c1; c += 4) {
        C x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = s_a[(c + u) * rp + tid];
#pragma unroll
        for (int t = 0; t < SW; ++t)
          if (t < usw) {
            C uu[4];
            ld4(&s_u[t][c], uu);
#pragma unroll
            for (int u = 0; u < 4; ++u) cfms(x[u], lv[t], uu[u]);
          }
#pragma unroll
        for (int u = 0; u < 4; ++u) s_a[(c + u) * rp + tid] = x[u];
      }
    } else {
      const int i = grow - ug0;
      for (int c = c0; c < c1; ++c) s_a[c * rp + tid] = s_u[i][c];
    }
  };

  for (int s0 = 0; s0 < w; s0 += SW) {
    const int sw = min(SW, w - s0), g0 = k + s0;
    const bool last = s0 + sw >= w;
#pragma unroll
    for (int c = 0; c < SW; ++c) v[c] = (grow != INT_MAX && c < sw) ? s_a[(s0 + c) * rp + tid] : czero;

#pragma unroll
    for (int jj = 0; jj < SW; ++jj) {  // unrolled: the register arrays are indexed statically
      if (jj >= sw) break;
      const int j = s0 + jj, gj = k + j, par = j & 1;
      const int owner = j / rp;
      if (amail && tid == 0) mbar_expect_tx(&s_mb[par], mail_bytes);  // arms this column's mailboxes
      // 1. Candidates: the best row of every warp stages its 8 values (and
      //    the thread holding row gj stages that row) before the CTA barrier.
      //    A NaN counts as 0, so every column has a pivot: row gj itself is
      //    always eligible.
      const bool elig = grow != INT_MAX && grow >= gj;
      R bv = R(-1);
      if (elig) {
        bv = cabs1(v[jj]);
        if (!(bv >= R(0))) bv = R(0);
      }
      if constexpr (sizeof(R) == 4) {
        // |re| + |im| >= 0, so its bits + 1 order as the value does (0: not
        // eligible) and the lowest lane, warp or CTA with the largest key
        // holds the first such row: one redux per level.
        const unsigned key = elig ? __float_as_uint(bv) + 1u : 0u;
        const unsigned mk = __reduce_max_sync(FULL, key);
        const int wl = __ffs(__ballot_sync(FULL, key == mk)) - 1;
        if (lane == wl && mk != 0u)
#pragma unroll
          for (int q = 0; q < KW; ++q) s_wt[par][warp][q] = row_word<R>(v, q);
        if (lane == 0) {
          s_rk[par][warp] = mk;
          s_rr[par][warp] = rbase + warp * 32 + wl;
        }
      } else {
        int br = elig ? grow : INT_MAX, bl = lane;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const R ov = __shfl_xor_sync(FULL, bv, off);
          const int orr = __shfl_xor_sync(FULL, br, off);
          const int ol = __shfl_xor_sync(FULL, bl, off);
          if (better(ov, orr, bv, br)) {
            bv = ov;
            br = orr;
            bl = ol;
          }
        }
        if (lane == bl && br != INT_MAX)
#pragma unroll
          for (int q = 0; q < KW; ++q) s_wt[par][warp][q] = row_word<R>(v, q);
        if (lane == 0) {
          s_rv[par][warp] = bv;
          s_rr[par][warp] = br;
        }
      }
      if (grow == gj)
#pragma unroll
        for (int q = 0; q < KW; ++q) s_gw[par][q] = row_word<R>(v, q);
      __syncthreads();
      // 2. The pushes, one 16-byte word per warp: word 0 is the candidate's
      //    (key or value, row), words 1..KW its values, the next KW row gj's
      //    (from its owner); every pushing warp finds this CTA's candidate.
      constexpr int NWORD = 1 + 2 * KW;
      if (warp < NWORD) {
        int cr, ww;
        uint4 cword;
        if constexpr (sizeof(R) == 4) {
          const unsigned ck = lane < NW ? s_rk[par][lane] : 0u;
          const unsigned mck = __reduce_max_sync(FULL, ck);
          ww = __ffs(__ballot_sync(FULL, lane < NW && ck == mck)) - 1;
          cr = mck ? s_rr[par][ww] : INT_MAX;
          cword = make_uint4(mck, 0u, (unsigned)cr, 0u);
        } else {
          R cv = lane < NW ? s_rv[par][lane] : R(-1);
          cr = lane < NW ? s_rr[par][lane] : INT_MAX;
          ww = lane;
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) {
            if (off >= NW) continue;
            const R ov = __shfl_xor_sync(FULL, cv, off);
            const int orr = __shfl_xor_sync(FULL, cr, off);
            const int ow = __shfl_xor_sync(FULL, ww, off);
            if (better(ov, orr, cv, cr)) {
              cv = ov;
              cr = orr;
              ww = ow;
            }
          }
          cv = __shfl_sync(FULL, cv, 0);
          cr = __shfl_sync(FULL, cr, 0);
          ww = __shfl_sync(FULL, ww, 0);
          cword = cand_word<R>(cv, cr);
        }
        if (lane < cs)
          for (int wi = warp; wi < NWORD; wi += NW) {
            if (amail) {  // every word goes out (the receiver counts bytes), row gj from its owner
              if (wi == 0)
                dsm_st4_async(&s_box[par][rank][0], lane, cword, &s_mb[par]);
              else if (wi <= KW)
                dsm_st4_async(&s_box[par][rank][wi], lane, s_wt[par][ww][wi - 1], &s_mb[par]);
              else if ((int)rank == owner)
                dsm_st4_async(&s_dbox[par][wi - 1 - KW], lane, s_gw[par][wi - 1 - KW], &s_mb[par]);
            } else if (wi == 0) {
              dsm_st4(&s_box[par][rank][0], lane, cword);
            } else if (wi <= KW) {
              if (cr != INT_MAX) dsm_st4(&s_box[par][rank][wi], lane, s_wt[par][ww][wi - 1]);
            } else if ((int)rank == owner) {
              dsm_st4(&s_dbox[par][wi - 1 - KW], lane, s_gw[par][wi - 1 - KW]);
            }
          }
      }
      if (amail) {
        // the column's mailboxes are full when the mbarrier's phase completes; a
        // wait that runs out sets the status and this thread skips its later
        // waits (the kernel still meets every cluster barrier), so a kernel
        // waits at most one limit in all.  No global read on this path: the
        // wait is on the critical path of every column.
        if (!gave_up && !mbar_wait(&s_mb[par], (mph >> par) & 1u, wlim)) {
          gave_up = true;
          atomicExch(&a.status[ST_TIMEOUT], 1);
        }
        mph ^= 1u << par;
      } else {
        cluster_sync();
      }
      // 3. The winner, by every warp from its own CTA's mailboxes.
      int prow, wsrc;
      if constexpr (sizeof(R) == 4) {
        const unsigned key = lane < cs ? s_box[par][lane][0].x : 0u;
        const unsigned mk = __reduce_max_sync(FULL, key);
        wsrc = __ffs(__ballot_sync(FULL, lane < cs && key == mk)) - 1;
        prow = (int)s_box[par][wsrc][0].z;
      } else {
        R wv = R(-1);
        int wr = INT_MAX, wk = lane;
        if (lane < cs) {
          const uint4 t0 = s_box[par][lane][0];
          wv = cand_val<R>(t0);
          wr = (int)t0.z;
        }
#pragma unroll
        for (int off = 8; off > 0; off >>= 1) {
          const R ov = __shfl_xor_sync(FULL, wv, off);
          const int orr = __shfl_xor_sync(FULL, wr, off);
          const int ok = __shfl_xor_sync(FULL, wk, off);
          if (better(ov, orr, wv, wr)) {
            wv = ov;
            wr = orr;
            wk = ok;
          }
        }
        prow = __shfl_sync(FULL, wr, 0);
        wsrc = __shfl_sync(FULL, wk, 0);
      }
      if (prow == INT_MAX || prow < gj) prow = gj;  // unreachable: row gj always takes part
      C piv[SW];
      row_unword<R>(&s_box[par][wsrc][1], piv);
      // 4. The interchange, on the sub-panel values in registers.
      if (prow != gj) {
        if (grow == prow) {
          row_unword<R>(&s_dbox[par][0], v);
        } else if (grow == gj) {
#pragma unroll
          for (int c = 0; c < SW; ++c) v[c] = piv[c];
        }
      }
#pragma unroll
      for (int c = 0; c < SW; ++c)
        if (c == jj) swp[c] = prow;
      if (tid < sw) s_u[jj][s0 + tid] = sel(piv, tid);  // the pivot row's L\U in the sub-panel
      // 5. Multipliers and the rank-1 update of the sub-panel, in registers.
      const C pj = piv[jj];
      const bool zero = pj.re == R(0) && pj.im == R(0);
      if (zero && rank == 0 && tid == 0 && !a.no_singular) atomicCAS(&a.status[ST_SINGULAR], 0, gj + 1);
      const C rpv = zero ? czero : crcp(pj);
      if (grow != INT_MAX && grow > gj) {
        const C l = v[jj] * rpv;
#pragma unroll
        for (int c = 0; c < SW; ++c) {
          if (c == jj) v[c] = l;
          if (c > jj) cfms(v[c], l, piv[c]);
        }
      }
    }
    // End of the sub-panel: registers back to shared memory.
    if (grow != INT_MAX)
#pragma unroll
      for (int c = 0; c < SW; ++c)
        if (c < sw) s_a[(s0 + c) * rp + tid] = v[c];
    // The sub-panel's interchanges as whole-row moves (position dst <- the
    // row at position src when the sub-panel started), by warp 0 of every
    // CTA: lane i holds touched position i and the start position of the row
    // now there.  Rank 0 also replays them on the panel's gather list.
    if (warp == 1 && rank == 0) {  // the gather list, beside warp 0's moves
      for (int jj = 0; jj < sw; ++jj) {
        const int j = s0 + jj, p = sel(swp, jj);
        {
          int ip = -1;
          if (p < k + w) {
            ip = p - k;
          } else {
            const int pc = s_pcount;
            for (int base = w; base < pc && ip < 0; base += 32) {
              const int e = base + lane;
              const unsigned m = __ballot_sync(FULL, e < pc && s_pdst[e] == p);
              if (m) ip = base + __ffs(m) - 1;
            }
            if (ip < 0) {
              ip = pc;
              if (lane == 0) {
                s_pdst[ip] = p;
                s_psrc[ip] = p;
                s_pcount = pc + 1;
              }
            }
            __syncwarp();
          }
          if (lane == 0) {
            s_ipiv[j] = p + 1;
            const int t = s_psrc[j];
            s_psrc[j] = s_psrc[ip];
            s_psrc[ip] = t;
          }
          __syncwarp();
        }
      }
    }
    if (warp == 0) {
      int pos = -1, lab = -1, n = 0;
      for (int jj = 0; jj < sw; ++jj) {
        const int tp = g0 + jj, p = sel(swp, jj);
        if (p != tp) {
          const unsigned mt = __ballot_sync(FULL, lane < n && pos == tp);
          int it = mt ? __ffs(mt) - 1 : -1;
          if (it < 0) {
            it = n++;
            if (lane == it) {
              pos = tp;
              lab = tp;
            }
          }
          const unsigned mp = __ballot_sync(FULL, lane < n && pos == p);
          int ipp = mp ? __ffs(mp) - 1 : -1;
          if (ipp < 0) {
            ipp = n++;
            if (lane == ipp) {
              pos = p;
              lab = p;
            }
          }
          const int lt = __shfl_sync(FULL, lab, it), lp = __shfl_sync(FULL, lab, ipp);
          if (lane == it) lab = lp;
          if (lane == ipp) lab = lt;
        }
      }
      // moves: touched positions whose row changed
      const bool mv = lane < n && lab != pos;
      const unsigned mm = __ballot_sync(FULL, mv);
      const int m = __popc(mm);
      int mslot = -1;
      if (mv) mslot = __popc(mm & ((1u << lane) - 1));
      // published rows: the move sources, then the pivot positions that keep
      // their row (their part right of the sub-panel is read from there)
      int pmove = -1;  // lane < sw: the move that fills pivot position g0 + lane
      {
        const unsigned md = __ballot_sync(FULL, mv && pos >= g0 && pos < g0 + sw);
        for (unsigned bits = md; bits; bits &= bits - 1) {
          const int l = __ffs(bits) - 1;
          const int d = __shfl_sync(FULL, pos, l), sl = __shfl_sync(FULL, mslot, l);
          if (lane == d - g0) pmove = sl;
        }
      }
      // move sources occupy entries 0..m-1 in move order
      const unsigned keep_piv = __ballot_sync(FULL, lane < sw && pmove < 0);
      if (mv) {
        s_mdst[mslot] = pos;
        s_msrc[mslot] = lab;
        s_ment[mslot] = mslot;
        s_ppos[mslot] = lab;
      }
      if (lane < sw) {
        if (pmove >= 0) {
          s_pent[lane] = pmove;
        } else {
          const int e = m + __popc(keep_piv & ((1u << lane) - 1));
          s_ppos[e] = g0 + lane;
          s_pent[lane] = e;
        }
      }
      if (lane == 0) {
        s_mcnt = m;
        s_pcnt = m + __popc(keep_piv);
      }
    }
    __syncthreads();
    // Publish: the part outside the sub-panel of every published row, as it
    // was when the sub-panel started (those columns have not changed since).
    const int npub = s_pcnt, nmov = s_mcnt;
    constexpr int PU = (kPushMoves * NB + NT - 1) / NT;
    {
      C t[PU];
      int off[PU];
#pragma unroll
      for (int u = 0; u < PU; ++u) {
        off[u] = -1;
        const int idx = tid + u * NT;
        if (idx < npub * w) {
          const int e = idx / w, c = idx % w, y = s_ppos[e];
          if (y >= rbase && y < rbase + rcount && (c < s0 || c >= s0 + sw)) {
            t[u] = s_a[(size_t)c * rp + (y - rbase)];
            off[u] = e * NB + c;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < PU; ++u)
        if (off[u] >= 0) s_pub[off[u]] = t[u];
    }
    cluster_sync();
    // Pull: rows of mine that receive another row, and (unless this is the
    // last sub-panel) the pivot rows' part right of the sub-panel; all remote
    // loads before the stores.
    {
      constexpr int UU = (SW * NB + NT - 1) / NT;
      C t[PU], tu[UU];
      int off[PU], offu[UU];
#pragma unroll
      for (int u = 0; u < PU; ++u) {
        off[u] = -1;
        const int idx = tid + u * NT;
        if (idx < nmov * w) {
          const int mi = idx / w, c = idx % w, x = s_mdst[mi];
          if (x >= rbase && x < rbase + rcount && (c < s0 || c >= s0 + sw)) {
            const int ys = s_msrc[mi];
            t[u] = dsm_ld(&s_pub[(size_t)s_ment[mi] * NB + c], (unsigned)((ys - k) / rp));
            off[u] = c * rp + (x - rbase);
          }
        }
      }
      const int wr = last ? 0 : w - s0 - sw;
#pragma unroll
      for (int u = 0; u < UU; ++u) {
        offu[u] = -1;
        const int idx = tid + u * NT;
        if (idx < sw * wr) {
          const int i = idx / wr, c = s0 + sw + idx % wr;
          const int e = s_pent[i], ys = s_ppos[e];
          tu[u] = dsm_ld(&s_pub[(size_t)e * NB + c], (unsigned)((ys - k) / rp));
          offu[u] = i * NB + c;
        }
      }
#pragma unroll
      for (int u = 0; u < PU; ++u)
        if (off[u] >= 0) s_a[off[u]] = t[u];
#pragma unroll
      for (int u = 0; u < UU; ++u)
        if (offu[u] >= 0) (&s_u[0][0])[offu[u]] = tu[u];
    }
    __syncthreads();
    if (last) break;
    // U of the pivot rows right of the sub-panel:
    // U(i,c) = A(i,c) - sum_{t<i} L(i,t) U(t,c), L = the sub-panel's unit lower.
    for (int c = s0 + sw + tid; c < w; c += NT)
      for (int i = 1; i < sw; ++i) {
        C x = s_u[i][c];
        for (int t = 0; t < i; ++t) cfms(x, s_u[i][s0 + t], s_u[t][c]);
        s_u[i][c] = x;
      }
    __syncthreads();
    if constexpr (sizeof(R) == 4) {
      // FP32 (the mixed form): the rank-8 product of the rows below the
      // pivot block on the tensor cores, as in the trailing update (TF32
      // operands, FP32 accumulation, subtracted in FP32): 16-row by 8-column
      // tiles, row tiles dealt round-robin to the warps.
      const int lo = max(0, g0 + sw - rbase);  // first local row to update
      const int mlo = lo & ~15;
      const int mtiles = rcount > lo ? (rcount - mlo + 15) / 16 : 0;
      const int c0 = s0 + sw, ntiles = (w - c0 + 7) / 8;
      const int g = lane >> 2, t4 = lane & 3;
      for (int mt = warp; mt < mtiles; mt += NW) {
        const int rb = mlo + mt * 16;
        const C x0 = s_a[(s0 + t4) * rp + rb + g], x1 = s_a[(s0 + t4) * rp + rb + g + 8];
        const C x2 = s_a[(s0 + t4 + 4) * rp + rb + g], x3 = s_a[(s0 + t4 + 4) * rp + rb + g + 8];
        const unsigned ar[4] = {to_tf32(x0.re), to_tf32(x1.re), to_tf32(x2.re), to_tf32(x3.re)};
        const unsigned ai[4] = {to_tf32(x0.im), to_tf32(x1.im), to_tf32(x2.im), to_tf32(x3.im)};
        const unsigned an[4] = {ai[0] ^ 0x80000000u, ai[1] ^ 0x80000000u, ai[2] ^ 0x80000000u,
                                ai[3] ^ 0x80000000u};
        for (int nt = 0; nt < ntiles; ++nt) {
          const int cb = c0 + nt * 8;
          const C y0 = s_u[t4][cb + g], y1 = s_u[t4 + 4][cb + g];
          const unsigned br[2] = {to_tf32(y0.re), to_tf32(y1.re)}, bi[2] = {to_tf32(y0.im), to_tf32(y1.im)};
          float pr[4] = {0.f, 0.f, 0.f, 0.f}, pi[4] = {0.f, 0.f, 0.f, 0.f};
          mma_tf32(pr, ar, br);
          mma_tf32(pr, an, bi);
          mma_tf32(pi, ar, bi);
          mma_tf32(pi, ai, br);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int lr = rb + g + ((e >> 1) << 3), c = cb + 2 * t4 + (e & 1);
            if (lr >= lo && lr < rcount) {
              C& z = s_a[c * rp + lr];
              z.re -= pr[e];
              z.im -= pi[e];
            }
          }
        }
      }
      if (grow != INT_MAX && grow >= g0 && grow < g0 + sw) {  // the pivot rows take their U
        const int i = grow - g0;
        for (int c = s0 + sw; c < w; ++c) s_a[c * rp + tid] = s_u[i][c];
      }
    } else {
      rank_update(v, g0, sw, s0 + sw, w);
    }
    __syncthreads();
  }
  for (int idx = tid; idx < w * rcount; idx += blockDim.x) {
    const int c = idx / rcount, r = idx % rcount;
    stc<R>(&A[(size_t)(k + c) * a.lda + rbase + r], s_a[c * rp + r]);
  }
  if (rank == 0) {
    if (tid < w) ipiv[k + tid] = s_ipiv[tid];
    if (tid == 0) perm[0] = s_pcount;
    for (int e = tid; e < s_pcount; e += blockDim.x) {
      perm[1 + 2 * e] = s_pdst[e];
      perm[2 + 2 * e] = s_psrc[e];
    }
  }
  cluster_sync();  // no CTA leaves while others may still read its shared memory
}

template <int NB, int NT>
__global__ void __launch_bounds__(NT, 1) k_panel_calu(PanelArgs a) {
  using C = zf;
  constexpr int SW = kCaluSW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_a = reinterpret_cast<C*>(smem_raw);  // [NB][rp] panel rows, column-major
  C* s_x = s_a + (size_t)NB * a.rp;          // [kCaluCand][SW] gathered candidates, then
                                             // [kCaluMoves][NB] published rows
  __shared__ __align__(16) C s_u[SW][NB];    // pivot rows: L\U in the block, A then U right of it
  __shared__ C s_lu[SW][SW];                 // the sub-panel's pivot block, L\U
  __shared__ C s_lv[SW][SW];                 // this CTA's candidates (values at the sub-panel start)
  __shared__ int s_lid[SW];                  // their positions (-1: none)
  __shared__ int s_cid[kCaluCand];
  __shared__ int s_pid[SW];                  // pivot rows (positions at the sub-panel start), in order
  __shared__ float s_rv[2][NT / 32];         // per-warp winners, double-buffered by step parity
  __shared__ int s_rr[2][NT / 32];
  __shared__ C s_wt[2][NT / 32][SW];         // ... and their current rows
  __shared__ C s_rcp[SW];                    // reciprocals of the pivot block's diagonal
  __shared__ int s_mdst[kCaluMoves], s_msrc[kCaluMoves], s_mcnt;
  __shared__ int s_ppos[kCaluMoves], s_pcnt;
  __shared__ int s_pdst[2 * NB], s_psrc[2 * NB];
  __shared__ int s_pcount;
  __shared__ int s_ipiv[NB];

  const unsigned rank = cluster_rank();
  const int prob = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float2* A = static_cast<float2*>(a.A) + (size_t)prob * a.bstride;
  int* ipiv = a.ipiv + (size_t)prob * a.ipiv_stride;
  int* perm = a.perm + (size_t)prob * a.perm_stride;
  const int rp = a.rp, w = a.w, k = a.k, cs = a.cs;
  const int rbase = k + (int)rank * rp;
  const int rcount = max(0, min(rp, a.nn - rbase));

  load_slice_async<float>(A, a.lda, rbase, k, rcount, w, s_a, rp);
  if (rank == 0 && prob == 0 && tid == 0 && a.pstart) {
    a.pstart[a.pidx] = k;
    a.pstart[a.pidx + 1] = k + w;
  }
  if (rank == 0 && tid < w) {
    s_pdst[tid] = k + tid;
    s_psrc[tid] = k + tid;
  }
  if (rank == 0 && tid == 0) s_pcount = w;
  __syncthreads();

  const int lr = tid;
  const int grow = lr < rcount ? rbase + lr : INT_MAX;
  C v[SW];
  auto zero = [] { return C{0.f, 0.f}; };

  for (int s0 = 0; s0 < w; s0 += SW) {
    const int sw = min(SW, w - s0);
    const int g0 = k + s0;
#pragma unroll
    for (int c = 0; c < SW; ++c) v[c] = (grow != INT_MAX && c < sw) ? s_a[(s0 + c) * rp + lr] : zero();
    const bool elig = grow != INT_MAX && grow >= g0;

    // 1. This CTA's candidates: partial pivoting on a copy of its rows, one
    //    barrier per column (each warp's winner stages its row before it).
    {
      constexpr int NW = NT / 32;
      C t[SW];
#pragma unroll
      for (int c = 0; c < SW; ++c) t[c] = v[c];
      bool chosen = false;
      for (int jj = 0; jj < sw; ++jj) {
        const int buf = jj & 1;
        float bv = -1.f;
        int br = INT_MAX;
        if (elig && !chosen) {
          bv = cabs1(sel(t, jj));
          if (!(bv >= 0.f)) bv = 0.f;  // a NaN still takes part, so a candidate always exists
          br = grow;
        }
        int bl = lane;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
          const int orr = __shfl_xor_sync(0xffffffffu, br, off);
          const int ol = __shfl_xor_sync(0xffffffffu, bl, off);
          if (better(ov, orr, bv, br)) {
            bv = ov;
            br = orr;
            bl = ol;
          }
        }
        if (br != INT_MAX && lane == bl) {
#pragma unroll
          for (int c = 0; c < SW; ++c) s_wt[buf][warp][c] = t[c];
        }
        if (lane == 0) {
          s_rv[buf][warp] = bv;
          s_rr[buf][warp] = br;
        }
        __syncthreads();
        float cv = lane < NW ? s_rv[buf][lane] : -1.f;
        int cr = lane < NW ? s_rr[buf][lane] : INT_MAX;
        int cw = lane;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          if (off >= NW) continue;
          const float ov = __shfl_xor_sync(0xffffffffu, cv, off);
          const int orr = __shfl_xor_sync(0xffffffffu, cr, off);
          const int ow = __shfl_xor_sync(0xffffffffu, cw, off);
          if (better(ov, orr, cv, cr)) {
            cv = ov;
            cr = orr;
            cw = ow;
          }
        }
        cr = __shfl_sync(0xffffffffu, cr, 0);
        cw = __shfl_sync(0xffffffffu, cw, 0);
        if (cr == INT_MAX) {
          if (tid == 0) s_lid[jj] = -1;
          continue;
        }
        if (grow == cr) {
          chosen = true;
#pragma unroll
          for (int c = 0; c < SW; ++c) s_lv[jj][c] = v[c];
          s_lid[jj] = cr;
        } else if (elig && !chosen) {
          const C* tw = s_wt[buf][cw];
          const C p = tw[jj];
          const C l = (p.re == 0.f && p.im == 0.f) ? zero() : sel(t, jj) * crcp(p);
#pragma unroll
          for (int c = 0; c < SW; ++c)
            if (c > jj) cfms(t[c], l, tw[c]);
        }
      }
    }
    cluster_sync();  // A: every CTA's candidates are published

    // 2. The cluster's candidates, the same partial pivoting in every CTA:
    //    4 warps, one candidate per thread, one named barrier per column.
    C* s_cv = s_x;
    for (int i = tid; i < cs * SW; i += NT) s_cid[i] = dsm_ld(&s_lid[i % SW], (unsigned)(i / SW));
    for (int i = tid; i < cs * SW * SW; i += NT) {
      const int cand = i / SW, c = i % SW;
      s_cv[i] = dsm_ld(&s_lv[cand % SW][c], (unsigned)(cand / SW));
    }
    __syncthreads();
    if (tid < kCaluCand) {
      const int cand = tid;
      const int id = (cand < cs * SW && (cand % SW) < sw) ? s_cid[cand] : -1;
      bool ch = false;
      C T[SW];
#pragma unroll
      for (int c = 0; c < SW; ++c) T[c] = id >= 0 ? s_cv[cand * SW + c] : zero();
      for (int jj = 0; jj < sw; ++jj) {
        const int buf = jj & 1;
        float bv = -1.f;
        int bid = INT_MAX;
        if (id >= 0 && !ch) {
          bv = cabs1(sel(T, jj));
          if (!(bv >= 0.f)) bv = 0.f;
          bid = id;
        }
        int bl = lane;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const float ov = __shfl_xor_sync(0xffffffffu, bv, off);
          const int oid = __shfl_xor_sync(0xffffffffu, bid, off);
          const int ol = __shfl_xor_sync(0xffffffffu, bl, off);
          if (better(ov, oid, bv, bid)) {
            bv = ov;
            bid = oid;
            bl = ol;
          }
        }
        if (bid != INT_MAX && lane == bl) {
#pragma unroll
          for (int c = 0; c < SW; ++c) s_wt[buf][warp][c] = T[c];
        }
        if (lane == 0) {
          s_rv[buf][warp] = bv;
          s_rr[buf][warp] = bid;
        }
        asm volatile("bar.sync 1, %0;" ::"n"(kCaluCand) : "memory");
        float fv = s_rv[buf][0];
        int fid = s_rr[buf][0], fw = 0;
#pragma unroll
        for (int q = 1; q < kCaluCand / 32; ++q)
          if (better(s_rv[buf][q], s_rr[buf][q], fv, fid)) {
            fv = s_rv[buf][q];
            fid = s_rr[buf][q];
            fw = q;
          }
        const C* tw = s_wt[buf][fw];
        if (id == fid) ch = true;
        if (tid == 0) {
          s_pid[jj] = fid;
#pragma unroll
          for (int c = 0; c < SW; ++c) s_lu[jj][c] = tw[c];
        }
        const C piv = tw[jj];
        const bool zp = piv.re == 0.f && piv.im == 0.f;
        if (zp && rank == 0 && tid == 0) atomicCAS(&a.status[ST_SINGULAR], 0, g0 + jj + 1);
        if (id >= 0 && !ch) {
          const C l = zp ? zero() : sel(T, jj) * crcp(piv);
#pragma unroll
          for (int c = 0; c < SW; ++c) {
            if (c == jj) T[c] = l;
            if (c > jj) cfms(T[c], l, tw[c]);
          }
        }
      }
    }
    __syncthreads();

    // 3. The interchanges in order (position of the pivot row swapped with
    //    position g0 + j), as position moves dst <- src (sub-panel start
    //    values), by warp 0: lane i holds touched position i and the start
    //    position of the row now there; the panel's gather list is updated
    //    the same way (rank 0).
    if (warp == 0) {
      int cur = lane < sw ? s_pid[lane] : -1;  // current position of pivot row `lane`
      int pos = -1, lab = -1, n = 0;
      for (int j = 0; j < sw; ++j) {
        const int tp = g0 + j, p = __shfl_sync(0xffffffffu, cur, j);
        if (rank == 0) {
          // the gather list: psrc[j'] <-> psrc[entry of position p]
          int ip = -1;
          if (p < k + w) {
            ip = p - k;
          } else {
            const int pc = s_pcount;
            for (int base = w; base < pc && ip < 0; base += 32) {
              const int e = base + lane;
              const unsigned m = __ballot_sync(0xffffffffu, e < pc && s_pdst[e] == p);
              if (m) ip = base + __ffs(m) - 1;
            }
            if (ip < 0) {
              ip = pc;
              if (lane == 0) {
                s_pdst[ip] = p;
                s_psrc[ip] = p;
                s_pcount = pc + 1;
              }
            }
            __syncwarp();
          }
          if (lane == 0) {
            s_ipiv[s0 + j] = p + 1;
            const int tmp = s_psrc[s0 + j];
            s_psrc[s0 + j] = s_psrc[ip];
            s_psrc[ip] = tmp;
          }
          __syncwarp();
        }
        if (p != tp) {
          unsigned mt = __ballot_sync(0xffffffffu, lane < n && pos == tp);
          int it = mt ? __ffs(mt) - 1 : -1;
          if (it < 0) {
            it = n++;
            if (lane == it) {
              pos = tp;
              lab = tp;
            }
          }
          unsigned mp = __ballot_sync(0xffffffffu, lane < n && pos == p);
          int ipp = mp ? __ffs(mp) - 1 : -1;
          if (ipp < 0) {
            ipp = n++;
            if (lane == ipp) {
              pos = p;
              lab = p;
            }
          }
          const int lt = __shfl_sync(0xffffffffu, lab, it), lp = __shfl_sync(0xffffffffu, lab, ipp);
          if (lane == it) lab = lp;
          if (lane == ipp) lab = lt;
          if (lane > j && lane < sw && cur == tp) cur = p;
        }
      }
      // moves: touched positions whose row changed
      const bool mv = lane < n && lab != pos;
      const unsigned mm = __ballot_sync(0xffffffffu, mv);
      if (mv) {
        const int slot = __popc(mm & ((1u << lane) - 1));
        s_mdst[slot] = pos;
        s_msrc[slot] = lab;
      }
      const int m = __popc(mm);
      // rows to publish: the pivot rows, then move sources not among them
      __syncwarp();
      const int cand_y = lane < sw ? s_pid[lane] : (lane < sw + m ? s_msrc[lane - sw] : -1);
      bool keep = cand_y >= 0;
      for (int i = 0; i < sw + m; ++i) {
        const int other = __shfl_sync(0xffffffffu, cand_y, i);
        if (i < lane && other == cand_y) keep = false;
      }
      const unsigned km = __ballot_sync(0xffffffffu, keep);
      if (keep) s_ppos[__popc(km & ((1u << lane) - 1))] = cand_y;
      if (lane == 0) {
        s_mcnt = m;
        s_pcnt = __popc(km);
      }
      if (lane < sw) {
        const C d = s_lu[lane][lane];
        s_rcp[lane] = (d.re == 0.f && d.im == 0.f) ? zero() : crcp(d);
      }
    }
    __syncthreads();

    // 4. Publish the rows that move or pivot, then pull the moved rows.
    C* s_pub = s_x;
    const int npub = s_pcnt, nmov = s_mcnt;
    for (int i = 0; i < npub; ++i) {
      const int y = s_ppos[i];
      if (y >= rbase && y < rbase + rcount) {
        const int ly = y - rbase;
        for (int c = tid; c < w; c += NT)
          if (c < s0 || c >= s0 + sw) s_pub[i * NB + c] = s_a[c * rp + ly];
        if (tid == ly)
#pragma unroll
          for (int c = 0; c < SW; ++c)
            if (c < sw) s_pub[i * NB + s0 + c] = v[c];
      }
    }
    cluster_sync();  // B: published rows visible
    auto pub_index = [&](int y) {
      int r = 0;
      for (int i = 0; i < npub; ++i)
        if (s_ppos[i] == y) r = i;
      return r;
    };
    for (int mv = 0; mv < nmov; ++mv) {
      const int x = s_mdst[mv];
      if (x >= rbase && x < rbase + rcount) {
        const int y = s_msrc[mv], pi = pub_index(y), lx = x - rbase;
        const unsigned owner = (unsigned)((y - k) / rp);
        for (int c = tid; c < w; c += NT)
          if (c < s0 || c >= s0 + sw) s_a[c * rp + lx] = dsm_ld(&s_pub[pi * NB + c], owner);
        if (tid == lx)
#pragma unroll
          for (int c = 0; c < SW; ++c)
            if (c < sw) v[c] = dsm_ld(&s_pub[pi * NB + s0 + c], owner);
      }
    }
    for (int idx = tid; idx < sw * w; idx += NT) {
      const int j = idx / w, c = idx % w;
      if (c >= s0 + sw) {
        const int y = s_pid[j];
        s_u[j][c] = dsm_ld(&s_pub[pub_index(y) * NB + c], (unsigned)((y - k) / rp));
      } else if (c >= s0) {
        s_u[j][c] = s_lu[j][c - s0];
      }
    }

    // 5. The sub-panel's L (and the pivot block) for my row.
    if (grow != INT_MAX && grow >= g0) {
      if (grow < g0 + sw) {
        const int j = grow - g0;
#pragma unroll
        for (int c = 0; c < SW; ++c) v[c] = s_lu[j][c];
      } else {
#pragma unroll
        for (int jj = 0; jj < SW; ++jj) {
          if (jj >= sw) break;
          C x = v[jj];
#pragma unroll
          for (int i = 0; i < jj; ++i) cfms(x, v[i], s_lu[i][jj]);
          v[jj] = x * s_rcp[jj];
        }
      }
    }
    // End of the sub-panel: registers back to shared memory.
    if (grow != INT_MAX)
#pragma unroll
      for (int c = 0; c < SW; ++c)
        if (c < sw) s_a[(s0 + c) * rp + lr] = v[c];
    __syncthreads();
    if (s0 + sw >= w) break;
    // U of the pivot rows right of the block:
    // U(i,c) = A(i,c) - sum_{t<i} L(i,t) U(t,c).
    for (int c = s0 + sw + tid; c < w; c += NT)
      for (int i = 1; i < sw; ++i) {
        C x = s_u[i][c];
        for (int t = 0; t < i; ++t) cfms(x, s_u[i][s0 + t], s_u[t][c]);
        s_u[i][c] = x;
      }
    __syncthreads();
    if (grow != INT_MAX && grow >= g0 + sw) {
      for (int c = s0 + sw; c < w; c += 4) {
        C x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = s_a[(c + u) * rp + lr];
#pragma unroll
        for (int t = 0; t < SW; ++t)
          if (t < sw) {
            C uu[4];
            ld4(&s_u[t][c], uu);
#pragma unroll
            for (int u = 0; u < 4; ++u) cfms(x[u], v[t], uu[u]);
          }
#pragma unroll
        for (int u = 0; u < 4; ++u) s_a[(c + u) * rp + lr] = x[u];
      }
    } else if (grow != INT_MAX && grow >= g0) {
      const int i = grow - g0;
      for (int c = s0 + sw; c < w; ++c) s_a[c * rp + lr] = s_u[i][c];
    }
    __syncthreads();
  }
  __syncthreads();
  for (int r = tid; r < rcount; r += NT)
    for (int c = 0; c < w; ++c) stc<float>(&A[(size_t)(k + c) * a.lda + rbase + r], s_a[c * rp + r]);
  if (rank == 0) {
    if (tid < w) ipiv[k + tid] = s_ipiv[tid];
    if (tid == 0) perm[0] = s_pcount;
    for (int e = tid; e < s_pcount; e += NT) {
      perm[1 + 2 * e] = s_pdst[e];
      perm[2 + 2 * e] = s_psrc[e];
    }
  }
  cluster_sync();  // no CTA leaves while others may still read its shared memory
}

// Fallback for panels too tall for one cluster: the same column steps over a
// cooperative grid of cs CTAs, exchanging candidates through global memory
// (double-buffered by column parity) with one bounded grid barrier per column.
template <typename R, int NB>
__global__ void __launch_bounds__(kPanelThreads) k_panel_grid(PanelArgs a) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_a = reinterpret_cast<C*>(smem_raw);
  __shared__ C s_piv[NB], s_drow[NB];
  __shared__ R s_rv[kPanelThreads / 32];
  __shared__ int s_rr[kPanelThreads / 32];
  __shared__ int s_best, s_win_row, s_win_cta;
  __shared__ int s_pdst[2 * NB], s_psrc[2 * NB];
  __shared__ int s_pcount;

  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned long long wlim = wait_limit(a.status);
  E* A = static_cast<E*>(a.A);
  const int rp = a.rp, w = a.w, k = a.k, G = a.cs;
  const int rbase = k + b * rp;
  const int rcount = max(0, min(rp, a.nn - rbase));
  R* slot_val = static_cast<R*>(a.slot_val);
  C* cand = static_cast<C*>(a.cand);
  C* drow = static_cast<C*>(a.drow);

  load_slice_async<R>(A, a.lda, rbase, k, rcount, w, s_a, rp);
  if (b == 0 && tid == 0 && a.pstart) {
    a.pstart[a.pidx] = k;
    a.pstart[a.pidx + 1] = k + w;
  }
  if (b == 0 && tid < w) {
    s_pdst[tid] = k + tid;
    s_psrc[tid] = k + tid;
  }
  if (b == 0 && tid == 0) s_pcount = w;
  __syncthreads();

  for (int j = 0; j < w; ++j) {
    const int gj = k + j, par = j & 1;
    R bv;
    int br;
    local_argmax<R>(s_a + j * rp, rcount, rbase, gj, s_rv, s_rr, bv, br);
    if (tid == 0) {
      slot_val[par * G + b] = bv;
      a.slot_row[par * G + b] = br;
      s_best = br;
    }
    __syncthreads();
    const int lbr = s_best;
    if (lbr != INT_MAX && tid < w) cand[((size_t)par * G + b) * NB + tid] = s_a[tid * rp + (lbr - rbase)];
    if (gj >= rbase && gj < rbase + rcount && tid < w) drow[par * NB + tid] = s_a[tid * rp + (gj - rbase)];
    if (!grid_barrier(a.bar, (unsigned)(j + 1), (unsigned)G, a.status, wlim)) return;
    if (tid == 0) __threadfence();
    if (warp == 0) {
      R v = R(-1);
      int rr = INT_MAX, cb = 0;
      for (int t = lane; t < G; t += 32) {
        const R tv = __ldcg(&slot_val[par * G + t]);
        const int tr = __ldcg(&a.slot_row[par * G + t]);
        if (better(tv, tr, v, rr)) {
          v = tv;
          rr = tr;
          cb = t;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const R ov = __shfl_xor_sync(0xffffffffu, v, off);
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
      s_piv[tid] = ldc_cg<R>(reinterpret_cast<const E*>(&cand[((size_t)par * G + pcta) * NB + tid]));
      s_drow[tid] = ldc_cg<R>(reinterpret_cast<const E*>(&drow[par * NB + tid]));
    }
    __syncthreads();
    if (prow != gj && prow >= rbase && prow < rbase + rcount && tid < w) s_a[tid * rp + (prow - rbase)] = s_drow[tid];
    if (gj >= rbase && gj < rbase + rcount && tid < w) s_a[tid * rp + (gj - rbase)] = s_piv[tid];
    if (b == 0 && tid == 0) {
      a.ipiv[gj] = prow + 1;
      perm_swap(s_pdst, s_psrc, s_pcount, k, w, j, prow);
    }
    __syncthreads();
    eliminate<R>(s_a, rp, rcount, rbase, gj, j, w, s_piv, a.status, b == 0);
  }
  for (int idx = tid; idx < w * rcount; idx += blockDim.x) {
    const int c = idx / rcount, r = idx % rcount;
    stc<R>(&A[(size_t)(k + c) * a.lda + rbase + r], s_a[c * rp + r]);
  }
  if (b == 0) {
    if (tid == 0) a.perm[0] = s_pcount;
    for (int e = tid; e < s_pcount; e += blockDim.x) {
      a.perm[1 + 2 * e] = s_pdst[e];
      a.perm[2 + 2 * e] = s_psrc[e];
    }
  }
}

// ---------------------------------------------------------------------------
// Tall FP32 panels by tournament pivoting (TSLU; option "panel_tslu").  A
// panel taller than one cluster holds (more than about 6900 rows of 64
// complex64 columns) is factored in three rounds instead of by the
// grid-barrier kernel, which pays a software grid barrier per column and takes
// the problems one at a time:
//   1. its rows are split into chunks of at most one cluster's rows; every
//      chunk (of every problem) is factored with partial pivoting by the
//      cluster kernel on a copy, in one launch, only to see which 64 rows it
//      picks;
//   2. those candidates (64 per chunk, their rows as they are in A) are
//      factored the same way: its 64 pivots are the panel's pivot rows;
//   3. the winners are brought to the top of the panel by the same sequence of
//      row interchanges partial pivoting would record (ipiv, gather list); the
//      top block is the winners' L11\U11 from round 2 (they were factored in
//      this order there) and L21 = A21 U11^-1.
// The factors satisfy A = P L U as every other panel's do, so the
// interchange, update and solve kernels are unchanged; the pivots may differ
// from per-column partial pivoting, which is why this is used for the FP32
// factors only (a preconditioner of the FP64 refinement).
// ---------------------------------------------------------------------------
constexpr int kTsluW = 64;

// Chunk c of problem b (rows k + c*chunk.. of the panel's 64 columns) into
// scratch problem b*nch + c, column-major chunk x 64; rows past nn are zero.
__global__ void __launch_bounds__(256) k_tslu_copy(const float2* __restrict__ Abase, size_t lda, size_t bstride,
                                                   int nn, int k, int chunk, int nch, float2* S) {
  const int c = blockIdx.y, b = blockIdx.z;
  const float2* A = Abase + (size_t)b * bstride;
  float2* Sp = S + (size_t)(b * nch + c) * chunk * kTsluW;
  const int r0 = k + c * chunk;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < chunk * kTsluW; idx += gridDim.x * blockDim.x) {
    const int col = idx / chunk, r = idx - col * chunk;
    const int gr = r0 + r;
    Sp[(size_t)col * chunk + r] = gr < nn ? A[(size_t)(k + col) * lda + gr] : make_float2(0.f, 0.f);
  }
}

// Candidate i = c*64 + e of problem b: the chunk row that chunk c's
// factorisation brought to its position e (entry e of its gather list), read
// from A as it is; cgid = that row's index in A, or -1 for a row past nn.
__global__ void __launch_bounds__(256) k_tslu_gather(const float2* __restrict__ Abase, size_t lda, size_t bstride,
                                                     int nn, int k, int chunk, int nch,
                                                     const int* __restrict__ cperm, float2* Cm, int* cgid) {
  const int b = blockIdx.y;
  const int ncand = nch * kTsluW;
  const float2* A = Abase + (size_t)b * bstride;
  float2* Cb = Cm + (size_t)b * ncand * kTsluW;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < ncand * kTsluW; idx += gridDim.x * blockDim.x) {
    const int col = idx / ncand, i = idx - col * ncand;
    const int c = i / kTsluW, e = i - c * kTsluW;
    const int src = cperm[(size_t)(b * nch + c) * kPermStride + 2 + 2 * e];
    const int g = k + c * chunk + src;
    const bool ok = g < nn;
    Cb[(size_t)col * ncand + i] = ok ? A[(size_t)(k + col) * lda + g] : make_float2(0.f, 0.f);
    if (col == 0) cgid[(size_t)b * ncand + i] = ok ? g : -1;
  }
}

// One CTA per problem: the winners (entries 0..63 of the candidates' gather
// list) become the pivot rows of columns k..k+63 in order, recorded as
// partial pivoting records them (ipiv, the panel's gather list); the panel's
// rows are interchanged accordingly and the top block takes the winners'
// L11\U11 from the candidates' factorisation.  Dynamic shared memory: the
// 128 x 64 interchanged rows.
__global__ void __launch_bounds__(256) k_tslu_apply(float2* Abase, size_t lda, size_t bstride, int nn, int k,
                                                    int ncand, const int* __restrict__ wperm,
                                                    const int* __restrict__ cgid, const float2* __restrict__ cfac,
                                                    int* ipiv, int ipiv_stride, int* perm, int* pstart, int pidx,
                                                    int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  zf* s_rows = reinterpret_cast<zf*>(smem_raw);       // [2*64][64]
  __shared__ int s_pdst[2 * kTsluW], s_psrc[2 * kTsluW];
  __shared__ int s_pcount;
  const int b = blockIdx.x, tid = threadIdx.x;
  float2* A = Abase + (size_t)b * bstride;
  const int* wp = wperm + (size_t)b * kPermStride;
  const int* gid = cgid + (size_t)b * ncand;
  int* pl = perm + (size_t)b * kPermStride;
  if (tid == 0) {
    int pcount = kTsluW;
    for (int e = 0; e < kTsluW; ++e) s_pdst[e] = s_psrc[e] = k + e;
    for (int j = 0; j < kTsluW; ++j) {
      const int g = gid[wp[2 + 2 * j]];
      int prow = k + j;  // no candidate row (past nn): the panel is singular there, keep the row
      if (g >= 0) {
        prow = g;  // where the winner's row is now: where an earlier interchange put it, else its own row
        for (int e = 0; e < pcount; ++e)
          if (s_psrc[e] == g) {
            prow = s_pdst[e];
            break;
          }
      }
      ipiv[(size_t)b * ipiv_stride + k + j] = prow + 1;
      perm_swap(s_pdst, s_psrc, pcount, k, kTsluW, j, prow);
    }
    s_pcount = pcount;
    pl[0] = pcount;
    if (b == 0 && pstart) {
      pstart[pidx] = k;
      pstart[pidx + 1] = k + kTsluW;
    }
  }
  __syncthreads();
  const int pc = s_pcount;
  for (int e = tid; e < pc; e += blockDim.x) {
    pl[1 + 2 * e] = s_pdst[e];
    pl[2 + 2 * e] = s_psrc[e];
  }
  // the interchanges on the panel's columns: every moved row read, then written
  for (int idx = tid; idx < pc * kTsluW; idx += blockDim.x) {
    const int e = idx / kTsluW, c = idx - e * kTsluW;
    const float2 v = A[(size_t)(k + c) * lda + s_psrc[e]];
    s_rows[e * kTsluW + c] = zf{v.x, v.y};
  }
  __syncthreads();
  for (int idx = tid; idx < pc * kTsluW; idx += blockDim.x) {
    const int e = idx / kTsluW, c = idx - e * kTsluW;
    const zf v = s_rows[e * kTsluW + c];
    if (e >= kTsluW) A[(size_t)(k + c) * lda + s_pdst[e]] = make_float2(v.re, v.im);
  }
  // rows k..k+63: L11\U11 of the winners in pivot order, which is the top
  // block of the candidates' factorisation (round 2) as it stands
  const float2* cf = cfac + (size_t)b * ncand * kTsluW;
  for (int idx = tid; idx < kTsluW * kTsluW; idx += blockDim.x) {
    const int c = idx / kTsluW, i = idx - c * kTsluW;
    const float2 v = cf[(size_t)c * ncand + i];
    A[(size_t)(k + c) * lda + k + i] = v;
    if (i == c && v.x == 0.f && v.y == 0.f) atomicCAS(&status[ST_SINGULAR], 0, k + c + 1);
  }
}

// L21 = A21 U11^-1 for rows k+64..nn-1 of problem blockIdx.y: one row per
// thread, its 64 values in registers, U11 (and the reciprocals of its
// diagonal) in shared memory.
__global__ void __launch_bounds__(128) k_tslu_trsm(float2* Abase, size_t lda, size_t bstride, int nn, int k) {
  __shared__ zf s_u[kTsluW][kTsluW + 1];
  __shared__ zf s_rd[kTsluW];
  float2* A = Abase + (size_t)blockIdx.y * bstride;
  for (int idx = threadIdx.x; idx < kTsluW * kTsluW; idx += blockDim.x) {
    const int c = idx / kTsluW, i = idx - c * kTsluW;
    const float2 v = A[(size_t)(k + c) * lda + k + i];
    s_u[i][c] = zf{v.x, v.y};
  }
  __syncthreads();
  if (threadIdx.x < kTsluW) {
    const zf d = s_u[threadIdx.x][threadIdx.x];
    s_rd[threadIdx.x] = (d.re == 0.f && d.im == 0.f) ? zf{0.f, 0.f} : crcp(d);
  }
  __syncthreads();
  for (int r = k + kTsluW + blockIdx.x * blockDim.x + threadIdx.x; r < nn; r += gridDim.x * blockDim.x) {
    zf x[kTsluW];
#pragma unroll
    for (int c = 0; c < kTsluW; ++c) {
      const float2 v = A[(size_t)(k + c) * lda + r];
      x[c] = zf{v.x, v.y};
    }
#pragma unroll
    for (int j = 0; j < kTsluW; ++j) {
      zf acc = x[j];
#pragma unroll
      for (int i = 0; i < j; ++i) cfms(acc, x[i], s_u[i][j]);
      x[j] = acc * s_rd[j];
    }
#pragma unroll
    for (int c = 0; c < kTsluW; ++c) A[(size_t)(k + c) * lda + r] = make_float2(x[c].re, x[c].im);
  }
}

// Row interchanges of one panel applied to columns [c0, ncols) as a gather,
// then U12 = L11^-1 A12 (unit lower).  One warp per column; problem = blockIdx.y.
// PRE: the previous panel (columns kprev..kprev+wprev-1, wprev = 16, 32, 48
// or 64) has not yet updated this panel's rows; its deferred product comes
// first.
template <typename R, bool PRE>
__global__ void __launch_bounds__(256) k_laswp_trsm(void* Av, size_t lda, size_t bstride, int k, int w, int c0,
                                                    int ncols, const int* __restrict__ perm, int perm_stride,
                                                    float* ure, float* uim, int urows, int ubase, int koff,
                                                    int kprev, int wprev) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  constexpr int NB = 64;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_L = reinterpret_cast<C*>(smem_raw);  // [NB][NB] column-major
  C* s_Lb = s_L + NB * NB;                  // PRE: the previous panel's L rows k..k+w-1 in this panel's order
  E* A = static_cast<E*>(Av) + (size_t)blockIdx.y * bstride;
  const int* pl = perm + (size_t)blockIdx.y * perm_stride;
  load_slice_async<R>(A, lda, k, k, w, w, s_L, NB);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int count = pl[0];
  pl += 1;
  if (PRE) {
    // s_Lb[j][i] = L(src(k + i), kprev + j): row k + i after this panel's
    // interchanges holds the old row src(k + i).  64 rows x 4 groups of 16
    // columns, all loads of a thread issued before its stores.
    const int i = threadIdx.x & 63, jg = threadIdx.x >> 6;
    if (i < w && jg * 16 < wprev) {
      const int src = pl[2 * i + 1];
      E t[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) t[u] = A[(size_t)(kprev + jg * 16 + u) * lda + src];
#pragma unroll
      for (int u = 0; u < 16; ++u) s_Lb[(jg * 16 + u) * NB + i] = C{t[u].x, t[u].y};
    }
  }
  __syncthreads();
  // The gather list is the same for every column: source rows of the panel
  // rows lane, lane+32, and (destination, source) of the displaced rows.
  const int s0 = lane < w ? pl[2 * lane + 1] : 0;
  const int s1 = lane + 32 < w ? pl[2 * (lane + 32) + 1] : 0;
  int xd[2], xs[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int e = w + lane + 32 * h;
    xd[h] = e < count ? pl[2 * e] : -1;
    xs[h] = e < count ? pl[2 * e + 1] : 0;
  }
  constexpr int QC = 4;  // columns per warp, solved as interleaved chains
  const int ncol = ncols - c0;
  for (int cb = (blockIdx.x * 8 + warp) * QC; cb < ncol; cb += gridDim.x * 8 * QC) {
    C v0[QC], v1[QC], x[QC][2], u0[QC], u1[QC];
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const bool ok = cb + q < ncol;
      const E* cp = A + (size_t)(c0 + cb + q) * lda;
      v0[q] = ok && lane < w ? ldc<R>(&cp[s0]) : C{R(0), R(0)};
      v1[q] = ok && lane + 32 < w ? ldc<R>(&cp[s1]) : C{R(0), R(0)};
#pragma unroll
      for (int h = 0; h < 2; ++h) x[q][h] = ok && xd[h] >= 0 ? ldc<R>(&cp[xs[h]]) : C{R(0), R(0)};
      if (PRE) {
        u0[q] = ok && lane < wprev ? ldc<R>(&cp[kprev + lane]) : C{R(0), R(0)};
        u1[q] = ok && lane + 32 < wprev ? ldc<R>(&cp[kprev + lane + 32]) : C{R(0), R(0)};
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      if (cb + q >= ncol) continue;
      E* cp = A + (size_t)(c0 + cb + q) * lda;
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (xd[h] >= 0) stc<R>(&cp[xd[h]], x[q][h]);
    }
    if (PRE) {
      // The previous panel's deferred update of this panel's rows:
      // v -= L(rows, kprev..kprev+wprev-1) U(kprev..kprev+wprev-1, col).
      for (int j = 0; j < wprev; ++j) {
        const C l0 = s_Lb[j * NB + lane], l1 = s_Lb[j * NB + lane + 32];
#pragma unroll
        for (int q = 0; q < QC; ++q) {
          const C src = (j < 32) ? u0[q] : u1[q];
          C uj;
          uj.re = __shfl_sync(0xffffffffu, src.re, j & 31);
          uj.im = __shfl_sync(0xffffffffu, src.im, j & 31);
          if (lane < w) cfms(v0[q], l0, uj);
          if (lane + 32 < w) cfms(v1[q], l1, uj);
        }
      }
    }
    // Forward substitution with the unit lower L11: rows lane and lane+32.
    for (int i = 0; i < w; ++i) {
      const C l0 = s_L[i * NB + lane], l1 = s_L[i * NB + lane + 32];
#pragma unroll
      for (int q = 0; q < QC; ++q) {
        const C src = (i < 32) ? v0[q] : v1[q];
        C ui;
        ui.re = __shfl_sync(0xffffffffu, src.re, i & 31);
        ui.im = __shfl_sync(0xffffffffu, src.im, i & 31);
        if (lane > i && lane < w) cfms(v0[q], l0, ui);
        if (lane + 32 > i && lane + 32 < w) cfms(v1[q], l1, ui);
      }
    }
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      if (cb + q >= ncol) continue;
      E* cp = A + (size_t)(c0 + cb + q) * lda;
      if (lane < w) stc<R>(&cp[k + lane], v0[q]);
      if (lane + 32 < w) stc<R>(&cp[k + lane + 32], v1[q]);
      if (ure) {
        // Packed K-major copies of U12 for the tensor-core update, rounded to TF32.
        const size_t row = ((size_t)blockIdx.y * urows + (c0 + cb + q - ubase)) * kTcKPitch + koff;
        const float r0 = lane < w ? (float)v0[q].re : 0.f, i0 = lane < w ? (float)v0[q].im : 0.f;
        const float r1 = lane + 32 < w ? (float)v1[q].re : 0.f, i1 = lane + 32 < w ? (float)v1[q].im : 0.f;
        unsigned t0, t1, t2, t3;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t0) : "f"(r0));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t1) : "f"(r1));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t2) : "f"(i0));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t3) : "f"(i1));
        ure[row + lane] = __uint_as_float(t0);
        ure[row + lane + 32] = __uint_as_float(t1);
        uim[row + lane] = __uint_as_float(t2);
        uim[row + lane + 32] = __uint_as_float(t3);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_laswp_tc: k_laswp_trsm for the FP32 factors on the tensor cores.  Each
// CTA first loads L11^-1 (k_l11_inv, once per panel), then loops over
// 64-column tiles of [c0, ncols): the tile's
// panel rows are gathered (the panel's interchanges), the displaced rows are
// copied down, PRE subtracts the previous panel's deferred product Lb Uprev,
// and U12 = L11^-1 B; both products as TF32 mma.sync (FP32 accumulation,
// complex as four real products): the deferred product in the accuracy class
// of the trailing update, U12 with split operands (3 x TF32, about FP32).  U12 goes back to A and, packed and rounded to
// TF32, to the tensor-core operand rows (ure/uim, when given).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = smem_u32(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned s = smem_u32(smem);
  const int n = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int kLtLd = 68;  // complex pitch of the 64 x 64 shared tiles (conflict-free fragment loads)
constexpr size_t kLtTile = (size_t)64 * kLtLd * sizeof(float2);

// L11^-1 of the panel at (k, k) (unit lower, w x w, zero-padded to 64 x 64)
// for k_laswp_tc, once per panel and problem (one CTA each): by 16 x 16
// diagonal blocks (a warp each, lane = column), then [[X11, 0], [X21, X22]]
// with X21 = -X22 L21 X11 at 16 and at 32 (one output per thread of 1024);
// the zero block above the diagonal (rows 0-31, columns 32-63) holds the
// intermediate L21 X11.  Row-major [64][64] per problem.
// In a group of gsize panels (panel gi of it, gi >= 0), it also keeps the
// group's row maps: map j (of the group's panel j < gsize - 1) gives, for a
// position x now, the position the row held after panel j (where L of panel
// j stores it). Panel gi replays its interchanges on maps j < gi and starts
// map gi as the identity below its rows.
__global__ void __launch_bounds__(1024) k_l11_inv(const float2* __restrict__ Abase, size_t lda, size_t bstride, int k,
                                                  int w, float2* out, const int* __restrict__ perm, int perm_stride,
                                                  int* gmap, int nn, int gi, int gsize) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_inv = reinterpret_cast<float2*>(smem_raw);  // [64][kLtLd]
  float2* s_b = s_inv + 64 * kLtLd;                      // [64][kLtLd] L11
  const int prob = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const float2* A = Abase + (size_t)prob * bstride;
  // L11 (unit lower, w x w at (k, k)) into registers first: these loads
  // overlap the row maps' dependent loads below
  float2 lv[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int idx = tid + q * 1024, i = idx & 63, c = idx >> 6;
    lv[q] = (i < w && c < w) ? A[(size_t)(k + c) * lda + k + i] : make_float2(0.f, 0.f);
  }
  if (gi >= 0) {
    int* gm = gmap + (size_t)prob * kGroupMaps * nn;
    const int* pl = perm + (size_t)prob * perm_stride;
    const int count = pl[0];
    const int j = tid >> 7, e = tid & 127;  // map j, entry e (at most 128 entries, 3 maps)
    int val = 0, dst = -1;
    if (j < gi && j < kGroupMaps && e < count) {
      val = gm[(size_t)j * nn + pl[2 + 2 * e]];
      dst = pl[1 + 2 * e];
    }
    __syncthreads();  // every read before any write
    if (dst >= 0) gm[(size_t)j * nn + dst] = val;
    if (gi < gsize - 1 && gi < kGroupMaps)
      for (int x = k + w + tid; x < nn; x += blockDim.x) gm[(size_t)gi * nn + x] = x;
  }
  // L11 into s_b, row-major; s_inv = I (1024 threads, 4 entries each)
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int idx = tid + q * 1024, i = idx & 63, c = idx >> 6;
    s_b[i * kLtLd + c] = lv[q];
    s_inv[i * kLtLd + c] = make_float2(i == c ? 1.f : 0.f, 0.f);
  }
  __syncthreads();
  // X = L11^-1 by blocks: the four 16 x 16 diagonal blocks (a warp each,
  // lane = column), then [[X11, 0], [X21, X22]] with X21 = -X22 L21 X11 at
  // 16 and at 32; the zero block above the diagonal (rows 0-31, columns
  // 32-63 of s_inv) holds the intermediate L21 X11.
  auto at = [&](float2* M, int i, int j) -> float2& { return M[i * kLtLd + j]; };
  if (warp < 4 && lane < 16) {
    const int b0 = 16 * warp, c = lane;
    zf x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = zf{i == c ? 1.f : 0.f, 0.f};
#pragma unroll
    for (int i = 1; i < 16; ++i) {
      zf acc{0.f, 0.f}, acc2{0.f, 0.f};  // two chains: even and odd t
#pragma unroll
      for (int t = 0; t < i; ++t) {  // x_t = 0 for t < c
        const float2 l = at(s_b, b0 + i, b0 + t);
        cfms((t & 1) ? acc2 : acc, zf{l.x, l.y}, x[t]);
      }
      if (i > c) x[i] = zf{acc.re + acc2.re, acc.im + acc2.im};
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) at(s_inv, b0 + i, b0 + c) = make_float2(x[i].re, x[i].im);
  }
  __syncthreads();
  // X21 = -X22 (L21 X11) for two 16-blocks (h = 16) and then one 32-block (h = 32)
  for (int h = 16; h <= 32; h *= 2) {
    const int npair = 64 / (2 * h), outs = npair * h * h;
    for (int idx = tid; idx < outs; idx += blockDim.x) {  // T = L21 X11 into the scratch block
      const int pp = idx / (h * h), i = (idx / h) % h, j = idx % h, o = pp * 2 * h;
      zf acc{0.f, 0.f}, acc2{0.f, 0.f};  // two chains: even and odd t
      for (int t = 0; t < h; t += 2) {
        const float2 l = at(s_b, o + h + i, o + t), x = at(s_inv, o + t, o + j);
        const float2 l2 = at(s_b, o + h + i, o + t + 1), x2 = at(s_inv, o + t + 1, o + j);
        cfms(acc, zf{l.x, l.y}, zf{x.x, x.y});
        cfms(acc2, zf{l2.x, l2.y}, zf{x2.x, x2.y});
      }
      at(s_inv, pp * h + i, 32 + j) = make_float2(-acc.re - acc2.re, -acc.im - acc2.im);  // acc = -T
    }
    __syncthreads();
    for (int idx = tid; idx < outs; idx += blockDim.x) {  // X21 = -X22 T
      const int pp = idx / (h * h), i = (idx / h) % h, j = idx % h, o = pp * 2 * h;
      zf acc{0.f, 0.f}, acc2{0.f, 0.f};
      for (int t = 0; t < h; t += 2) {
        const float2 x = at(s_inv, o + h + i, o + h + t), tt = at(s_inv, pp * h + t, 32 + j);
        const float2 x2 = at(s_inv, o + h + i, o + h + t + 1), tt2 = at(s_inv, pp * h + t + 1, 32 + j);
        cfms(acc, zf{x.x, x.y}, zf{tt.x, tt.y});
        cfms(acc2, zf{x2.x, x2.y}, zf{tt2.x, tt2.y});
      }
      at(s_inv, o + h + i, o + j) = make_float2(acc.re + acc2.re, acc.im + acc2.im);  // acc = -X22 T
    }
    __syncthreads();
  }
  for (int idx = tid; idx < 32 * 32; idx += blockDim.x) at(s_inv, idx >> 5, 32 + (idx & 31)) = make_float2(0.f, 0.f);
  __syncthreads();
  float2* o = out + (size_t)prob * 64 * 64;
  for (int idx = tid; idx < 64 * 64; idx += blockDim.x) o[idx] = s_inv[(idx >> 6) * kLtLd + (idx & 63)];
}

template <bool PRE>
__global__ void __launch_bounds__(256, 1) k_laswp_tc(float2* Abase, size_t lda, size_t bstride, int k, int w, int c0,
                                                     int ncols, const int* __restrict__ perm, int perm_stride,
                                                     float* ure, float* uim, int urows, int ubase, int koff,
                                                     int kfirst, int nprev, int cdefer, const int* __restrict__ gmap,
                                                     int nn, const float2* __restrict__ linv, float* lhat, int lrows,
                                                     int pk_r0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_inv = reinterpret_cast<float2*>(smem_raw);  // [64][kLtLd] L11^-1, row-major
  float2* s_bb = s_inv + 64 * kLtLd;                     // [2][64][kLtLd] tiles (panel rows x columns), two stages
  float2* s_lb = s_bb + 2 * 64 * kLtLd;                  // PRE: an earlier panel's L at this panel's rows
  float2* s_upb = s_lb + 64 * kLtLd;                     // PRE: [2][64][kLtLd] that panel's U rows of the tile
  __shared__ int s_src[64];                              // source row of panel row i
  __shared__ int s_xd[64], s_xs[64];                     // displaced rows: dst <- src
  __shared__ int s_nx;
  const int prob = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float2* A = Abase + (size_t)prob * bstride;
  const int* pl = perm + (size_t)prob * perm_stride;
  const int count = pl[0];
  if (tid < 64) s_src[tid] = tid < w ? pl[2 + 2 * tid] : 0;
  if (tid < 64) {
    const int e = w + tid;
    s_xd[tid] = e < count ? pl[1 + 2 * e] : -1;
    s_xs[tid] = e < count ? pl[2 + 2 * e] : 0;
  }
  if (tid == 0) s_nx = max(0, count - w);
  // L11^-1 (k_l11_inv) into s_inv by cp.async
  {
    const float2* li = linv + (size_t)prob * 64 * 64;
    for (int idx = tid; idx < 64 * 64; idx += blockDim.x)
      cp_async8(&s_inv[(idx >> 6) * kLtLd + (idx & 63)], &li[idx], true);
    cp_async_commit();
  }
  __syncthreads();  // s_src
  // Lb_j(i, t) = L(map_j(k + i), kfirst + 64 j + t): earlier panel j's L at this panel's rows
  const int* gm = gmap + (size_t)prob * kGroupMaps * nn;
  auto load_lb_to = [&](float2* dst, int j) {
    for (int idx = tid; idx < 64 * 64; idx += blockDim.x) {
      const int i = idx & 63, t = idx >> 6;
      const bool ok = i < w;
      cp_async8(&dst[i * kLtLd + t], ok ? &A[(size_t)(kfirst + 64 * j + t) * lda + gm[(size_t)j * nn + k + i]] : A,
                ok);
    }
  };
  auto load_lb = [&](int j) { load_lb_to(s_lb, j); };
  // earlier panel j's U rows of the tile at cbase (tw columns)
  auto load_up_to = [&](float2* dst, int j, int cbase, int tw) {
    const int i = tid & 63, cg = tid >> 6;
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int c = cg + 4 * u;
      cp_async8(&dst[i * kLtLd + c], c < tw ? &A[(size_t)(cbase + c) * lda + kfirst + 64 * j + i] : A, c < tw);
    }
  };
  if (PRE) load_lb(0);
  cp_async_commit();

  // warp tile: rows [16 * (warp & 3), +16) x columns [32 * (warp >> 2), +32)
  const int g = lane >> 2, t4 = lane & 3, mrow = 16 * (warp & 3), ncol = 32 * (warp >> 2);
  // acc += M B for this warp's tile, M (64 x 64) and B (64 x 64) complex in
  // shared memory; split: each operand as a TF32 pair hi + lo and three
  // products per real product (hi hi + hi lo + lo hi), about FP32 accuracy.
  auto zero_acc = [&](float (&pr)[4][4], float (&pi)[4][4]) {
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) pr[nt][e] = pi[nt][e] = 0.f;
  };
  auto cproduct = [&](const float2* M, const float2* Bm, float (&pr)[4][4], float (&pi)[4][4], bool split) {
#pragma unroll 2
    for (int ks = 0; ks < 8; ++ks) {
      const int kc = ks * 8 + t4;
      const float2 x0 = M[(mrow + g) * kLtLd + kc], x1 = M[(mrow + g + 8) * kLtLd + kc];
      const float2 x2 = M[(mrow + g) * kLtLd + kc + 4], x3 = M[(mrow + g + 8) * kLtLd + kc + 4];
      const unsigned ar[4] = {to_tf32(x0.x), to_tf32(x1.x), to_tf32(x2.x), to_tf32(x3.x)};
      const unsigned ai[4] = {to_tf32(x0.y), to_tf32(x1.y), to_tf32(x2.y), to_tf32(x3.y)};
      const unsigned an[4] = {ai[0] ^ 0x80000000u, ai[1] ^ 0x80000000u, ai[2] ^ 0x80000000u, ai[3] ^ 0x80000000u};
      unsigned arl[4], ail[4], anl[4];  // low parts (split)
      if (split) {
        const float xr[4] = {x0.x, x1.x, x2.x, x3.x}, xi[4] = {x0.y, x1.y, x2.y, x3.y};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          arl[e] = to_tf32(xr[e] - __uint_as_float(ar[e]));
          ail[e] = to_tf32(xi[e] - __uint_as_float(ai[e]));
          anl[e] = ail[e] ^ 0x80000000u;
        }
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int cb = ncol + nt * 8 + g;
        const float2 y0 = Bm[kc * kLtLd + cb], y1 = Bm[(kc + 4) * kLtLd + cb];
        const unsigned br[2] = {to_tf32(y0.x), to_tf32(y1.x)}, bi[2] = {to_tf32(y0.y), to_tf32(y1.y)};
        mma_tf32(pr[nt], ar, br);
        mma_tf32(pr[nt], an, bi);
        mma_tf32(pi[nt], ar, bi);
        mma_tf32(pi[nt], ai, br);
        if (split) {
          const unsigned brl[2] = {to_tf32(y0.x - __uint_as_float(br[0])), to_tf32(y1.x - __uint_as_float(br[1]))};
          const unsigned bil[2] = {to_tf32(y0.y - __uint_as_float(bi[0])), to_tf32(y1.y - __uint_as_float(bi[1]))};
          mma_tf32(pr[nt], ar, brl);
          mma_tf32(pr[nt], an, bil);
          mma_tf32(pi[nt], ar, bil);
          mma_tf32(pi[nt], ai, brl);
          mma_tf32(pr[nt], arl, br);
          mma_tf32(pr[nt], anl, bi);
          mma_tf32(pi[nt], arl, bi);
          mma_tf32(pi[nt], ail, br);
        }
      }
    }
  };

  const int ntiles = (ncols - c0 + 63) / 64;
  // A tile's gathered panel rows into stage st by cp.async (8-byte elements,
  // zero-filled outside the panel rows and past the last column).
  // With it, for a deferred tile, the first earlier panel's U rows (and its
  // Lb again when the tile before used s_lb for a third panel).
  auto issue = [&](int tile, int st, bool lb0) {
    if (tile < ntiles) {
      const int cbase = c0 + tile * 64, tw = min(64, ncols - cbase);
      float2* b = s_bb + (size_t)st * 64 * kLtLd;
      const int i = tid & 63, cg = tid >> 6;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int c = cg + 4 * u;
        const bool ok = c < tw && i < w;
        cp_async8(&b[i * kLtLd + c], ok ? &A[(size_t)(cbase + c) * lda + s_src[i]] : A, ok);
      }
      if (PRE && cbase >= cdefer) {
        load_up_to(s_upb + (size_t)st * 64 * kLtLd, 0, cbase, tw);
        if (lb0) load_lb(0);
      }
    }
    cp_async_commit();
  };
  issue(blockIdx.x, 0, false);
  for (int it = 0;; ++it) {
    const int tile = blockIdx.x + it * gridDim.x;
    if (tile >= ntiles) break;
    const int st = it & 1;
    const int cbase = c0 + tile * 64, tw = min(64, ncols - cbase);
    float2* sb = s_bb + (size_t)st * 64 * kLtLd;
    cp_async_wait<0>();
    __syncthreads();
    // displaced rows: their sources, loaded now and stored after the products
    float2 xv[16];
    const int nx = s_nx;
    {
      const int i = tid & 63, cg = tid >> 6;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int c = cg + 4 * u;
        xv[u] = (i < nx && c < tw) ? A[(size_t)(cbase + c) * lda + s_xs[i]] : make_float2(0.f, 0.f);
      }
    }
    float pr[4][4], pi[4][4];
    if (PRE && cbase >= cdefer) {  // B -= sum_j Lb_j Uprev_j: the group's deferred update of these rows
      // Two operand slots: slot 0 = (s_lb, this stage's U buffer), which the
      // tile's own loads filled with panel 0's; slot 1 = the other stage's
      // tile and U buffers, idle until the next tile is issued.  Panel j + 1's
      // operands load into the other slot while panel j's product runs.
      float2* const lb0 = s_lb;
      float2* const lb1 = s_bb + (size_t)(st ^ 1) * 64 * kLtLd;
      float2* const up0 = s_upb + (size_t)st * 64 * kLtLd;
      float2* const up1 = s_upb + (size_t)(st ^ 1) * 64 * kLtLd;
      zero_acc(pr, pi);
      for (int j = 0; j < nprev; ++j) {
        const bool odd = j & 1;
        if (j + 1 < nprev) {
          load_lb_to(odd ? lb0 : lb1, j + 1);
          load_up_to(odd ? up0 : up1, j + 1, cbase, tw);
          cp_async_commit();
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncthreads();
        cproduct(odd ? lb1 : lb0, odd ? up1 : up0, pr, pi, false);
        __syncthreads();  // slot sl is refilled two panels on
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int r = mrow + g + ((e >> 1) << 3), c = ncol + nt * 8 + 2 * t4 + (e & 1);
          float2& z = sb[r * kLtLd + c];
          z.x -= pr[nt][e];
          z.y -= pi[nt][e];
        }
      __syncthreads();
    }
    issue(tile + gridDim.x, st ^ 1, nprev >= 3);  // the next tile streams in meanwhile
    zero_acc(pr, pi);
    cproduct(s_inv, sb, pr, pi, true);  // U12 = L11^-1 B
    __syncthreads();                     // every warp has read the tile
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = mrow + g + ((e >> 1) << 3), c = ncol + nt * 8 + 2 * t4 + (e & 1);
        sb[r * kLtLd + c] = make_float2(pr[nt][e], pi[nt][e]);
      }
    {  // displaced rows get the rows they replaced (all reads of them came first)
      const int i = tid & 63, cg = tid >> 6;
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int c = cg + 4 * u;
        if (i < nx && c < tw) A[(size_t)(cbase + c) * lda + s_xd[i]] = xv[u];
      }
    }
    __syncthreads();
    {  // U12 to A (rows k..k+w-1) and packed K-major TF32 rows
      const int i = tid & 63, cg = tid >> 6;
#pragma unroll 4
      for (int u = 0; u < 16; ++u) {
        const int c = cg + 4 * u;
        if (c >= tw) continue;
        const float2 z = sb[i * kLtLd + c];
        if (i < w) A[(size_t)(cbase + c) * lda + k + i] = z;
        if (ure) {
          const size_t row = ((size_t)prob * urows + (cbase + c - ubase)) * kTcKPitch + koff;
          ure[row + i] = __uint_as_float(to_tf32(i < w ? z.x : 0.f));
          uim[row + i] = __uint_as_float(to_tf32(i < w ? z.y : 0.f));
        }
      }
    }
    __syncthreads();  // this stage is refilled two tiles on
  }
  cp_async_wait<0>();
  if (pk_r0 >= 0 && pk_r0 < nn) {
    // this panel's L21 (rows pk_r0..nn-1) packed for the update that follows,
    // at its K slot, 32-row blocks dealt to the CTAs (the tiles' shared memory)
    __shared__ int s_psrc[32];
    __syncthreads();
    auto tile = reinterpret_cast<float2(*)[33]>(s_bb);
    float* out = lhat + (size_t)prob * lrows * kTcKPitch;
    const int nblk = (nn - pk_r0 + 31) / 32;
    for (int bi = blockIdx.x; bi < nblk; bi += gridDim.x) {
      pack_l_rows(A, lda, nn, k, w, pk_r0, pk_r0 + 32 * bi, koff, out, nullptr, tile, s_psrc);
      __syncthreads();
    }
  }
}
// ---------------------------------------------------------------------------
// Trailing update C -= L21 U12 on the tensor cores, complex as 4 real products.
// C: rows [r0, nn), cols [c0, ncols) of problem blockIdx.z; L21 = columns
// k..k+w-1 of the same rows; U12 = rows k..k+w-1 of the same columns.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// FP64: CTA tile 64x64 complex, 8 warps of 32x16, k chunks of 16 double-buffered
// through cp.async.  As[k][m] (row stride 66) and Bs[n][k] (stride 20), in
// complex units, keep every fragment load conflict-free.
constexpr int GBM = 64, GBN = 64, GBK = 16;
constexpr int AS_STRIDE = GBM + 2;  // == 2 mod 8
constexpr int BS_STRIDE = GBK + 4;  // == 4 mod 8
constexpr size_t kGemmSmem = (size_t)2 * (GBK * AS_STRIDE + GBN * BS_STRIDE) * sizeof(double2);

// With gperm (a panel pair of the plain LU): the first wg of the K columns
// are the earlier panel's L, whose rows have not taken the later panel's
// interchanges; row r of C reads them at the row the later panel's gather
// list moved to r (count, then dst/src pairs; problem z's list at
// gperm + z * gperm_stride).
__global__ void __launch_bounds__(256, 2) k_gemm_f64(double2* Abase, size_t lda, size_t bstride, int nn, int k, int w,
                                                  int r0, int c0, int ncols, const int* __restrict__ gperm,
                                                  int gperm_stride, int wg) {
  extern __shared__ __align__(16) double2 g_smem[];
  auto As = reinterpret_cast<double2(*)[GBK][AS_STRIDE]>(g_smem);
  auto Bs = reinterpret_cast<double2(*)[GBN][BS_STRIDE]>(g_smem + 2 * GBK * AS_STRIDE);
  __shared__ int s_map[GBM];  // storage row of the gathered L columns for each tile row
  double2* A = Abase + (size_t)blockIdx.z * bstride;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps
  const int row0 = r0 + blockIdx.x * GBM, col0 = c0 + blockIdx.y * GBN;

  // The tile of C is read at the end: start bringing it into L2 now.
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int gr = row0 + wm * 32 + mt * 8 + g, gc = col0 + wn * 16 + nt * 8 + 2 * t + e;
        if (gr < nn && gc < ncols) asm volatile("prefetch.global.L2 [%0];" ::"l"(&A[(size_t)gc * lda + gr]));
      }
  if (tid < GBM) s_map[tid] = row0 + tid;
  __syncthreads();
  if (gperm && wg > 0) {
    const int* pl = gperm + (size_t)blockIdx.z * gperm_stride;
    const int cnt = pl[0];
    for (int e = tid; e < cnt; e += blockDim.x) {
      const int dst = pl[1 + 2 * e];
      if (dst >= row0 && dst < row0 + GBM) s_map[dst - row0] = pl[2 + 2 * e];
    }
  }
  __syncthreads();

  auto load_chunk = [&](int stage, int kc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int kk = idx >> 6, m = idx & 63;
      const int gr = row0 + m, gk = kc + kk;
      const bool ok = gr < nn && gk < w;
      const int sr = gk < wg ? s_map[m] : gr;
      cp_async16(&As[stage][kk][m], ok ? &A[(size_t)(k + gk) * lda + sr] : A, ok);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int n = idx >> 4, kk = idx & 15;
      const int gc = col0 + n, gk = kc + kk;
      const bool ok = gc < ncols && gk < w;
      cp_async16(&Bs[stage][n][kk], ok ? &A[(size_t)gc * lda + k + gk] : A, ok);
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
      // four passes over the 8 tiles: an accumulator's next product is 16
      // independent DMMAs away (each still takes its terms in the same order)
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma(acc_re[mt][nt][0], acc_re[mt][nt][1], af[mt].x, bf[nt].x);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma(acc_im[mt][nt][0], acc_im[mt][nt][1], af[mt].x, bf[nt].y);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma(acc_re[mt][nt][0], acc_re[mt][nt][1], -af[mt].y, bf[nt].y);
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) dmma(acc_im[mt][nt][0], acc_im[mt][nt][1], af[mt].y, bf[nt].x);
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

// FP32 storage, TF32 tensor cores (mma.sync m16n8k8, operands rounded to
// TF32, FP32 accumulation).  CTA tile 128x64 complex, 8 warps of 32x32,
// k chunks of 16.  As[k][m] row stride 136 float2 and Bs[n][k] stride 20.
constexpr int TBM = 128, TBN = 64, TBK = 16;
constexpr int TAS = TBM + 8;   // float2 units
constexpr int TBS = TBK + 4;
constexpr size_t kGemmTf32Smem = (size_t)2 * (TBK * TAS + TBN * TBS) * sizeof(float2);


__global__ void __launch_bounds__(256) k_gemm_tf32(float2* Abase, size_t lda, size_t bstride, int nn, int k, int w,
                                                   int r0, int c0, int ncols) {
  extern __shared__ __align__(16) float2 t_smem[];
  auto As = reinterpret_cast<float2(*)[TBK][TAS]>(t_smem);
  auto Bs = reinterpret_cast<float2(*)[TBN][TBS]>(t_smem + 2 * TBK * TAS);
  float2* A = Abase + (size_t)blockIdx.z * bstride;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 1, wn = warp & 1;  // 4 x 2 warps of 32x32
  const int row0 = r0 + blockIdx.x * TBM, col0 = c0 + blockIdx.y * TBN;

  auto load_chunk = [&](int stage, int kc) {
    // A: 16 k x 128 rows = 2048 float2, 8 per thread.
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int idx = tid + q * 256;
      const int kk = idx >> 7, m = idx & 127;
      const int gr = row0 + m, gk = kc + kk;
      const bool ok = gr < nn && gk < w;
      cp_async8(&As[stage][kk][m], ok ? &A[(size_t)(k + gk) * lda + gr] : A, ok);
    }
    // B: 64 cols x 16 k = 1024 float2, 4 per thread.
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * 256;
      const int n = idx >> 4, kk = idx & 15;
      const int gc = col0 + n, gk = kc + kk;
      const bool ok = gc < ncols && gk < w;
      cp_async8(&Bs[stage][n][kk], ok ? &A[(size_t)gc * lda + k + gk] : A, ok);
    }
    cp_async_commit();
  };

  float acc_re[2][4][4], acc_im[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc_re[i][j][e] = acc_im[i][j][e] = 0.f;

  const int nchunks = (w + TBK - 1) / TBK;
  load_chunk(0, 0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks) {
      load_chunk((c + 1) & 1, (c + 1) * TBK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int st = c & 1;
#pragma unroll
    for (int ks = 0; ks < TBK / 8; ++ks) {
      unsigned ar[2][4], ai[2][4], an[2][4], br_[4][2], bi[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int rb = wm * 32 + mt * 16 + g;
        const float2 x0 = As[st][ks * 8 + t][rb];
        const float2 x1 = As[st][ks * 8 + t][rb + 8];
        const float2 x2 = As[st][ks * 8 + t + 4][rb];
        const float2 x3 = As[st][ks * 8 + t + 4][rb + 8];
        ar[mt][0] = to_tf32(x0.x);
        ar[mt][1] = to_tf32(x1.x);
        ar[mt][2] = to_tf32(x2.x);
        ar[mt][3] = to_tf32(x3.x);
        ai[mt][0] = to_tf32(x0.y);
        ai[mt][1] = to_tf32(x1.y);
        ai[mt][2] = to_tf32(x2.y);
        ai[mt][3] = to_tf32(x3.y);
#pragma unroll
        for (int e = 0; e < 4; ++e) an[mt][e] = ai[mt][e] ^ 0x80000000u;
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int cb = wn * 32 + nt * 8 + g;
        const float2 y0 = Bs[st][cb][ks * 8 + t];
        const float2 y1 = Bs[st][cb][ks * 8 + t + 4];
        br_[nt][0] = to_tf32(y0.x);
        br_[nt][1] = to_tf32(y1.x);
        bi[nt][0] = to_tf32(y0.y);
        bi[nt][1] = to_tf32(y1.y);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          mma_tf32(acc_re[mt][nt], ar[mt], br_[nt]);
          mma_tf32(acc_re[mt][nt], an[mt], bi[nt]);
          mma_tf32(acc_im[mt][nt], ar[mt], bi[nt]);
          mma_tf32(acc_im[mt][nt], ai[mt], br_[nt]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int gr = row0 + wm * 32 + mt * 16 + g + ((e >> 1) << 3);
        const int gc = col0 + wn * 32 + nt * 8 + 2 * t + (e & 1);
        if (gr < nn && gc < ncols) {
          float2* p = &A[(size_t)gc * lda + gr];
          float2 v = *p;
          v.x -= acc_re[mt][nt][e];
          v.y -= acc_im[mt][nt][e];
          *p = v;
        }
      }
}

// ---------------------------------------------------------------------------
// Back substitution U x = y (y = column nn of A after the factorisation).
// Launch s handles block s (rows [s*64, ...)): every row above block s+1
// subtracts U(row, block s+1) x_{s+1}; CTA 0 owns the rows of block s, stages
// the block's upper triangle in shared memory and solves it.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_backsub(void* Av, size_t lda, size_t bstride, int nn, int s, void* yv,
                                                 size_t ystride) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  constexpr int NB = 64;
  __shared__ C s_x[NB];
  __shared__ C s_y[NB];
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_U = reinterpret_cast<C*>(smem_raw);  // column-major diagonal block (CTA 0)
  E* A = static_cast<E*>(Av) + (size_t)blockIdx.y * bstride;
  // The right-hand side: column nn of A, or a separate vector per problem.
  E* y = yv ? static_cast<E*>(yv) + (size_t)blockIdx.y * ystride : A + (size_t)nn * lda;
  const int b0 = s * NB, b1 = min(b0 + NB, nn);
  const int n0 = b1, n1 = min(b1 + NB, nn);
  const int wn = n1 - n0, wb = b1 - b0;
  for (int i = threadIdx.x; i < wn; i += blockDim.x) s_x[i] = ldc<R>(&y[n0 + i]);
  if (blockIdx.x == 0)
    for (int idx = threadIdx.x; idx < wb * wb; idx += blockDim.x) {
      const int c = idx / wb, r = idx % wb;
      s_U[c * NB + r] = ldc<R>(&A[(size_t)(b0 + c) * lda + b0 + r]);
    }
  __syncthreads();
  int lo, hi;
  if (blockIdx.x == 0) {
    lo = b0;
    hi = b1;
  } else {
    lo = (blockIdx.x - 1) * blockDim.x;
    hi = min(lo + (int)blockDim.x, b0);
  }
  const int r = lo + threadIdx.x;
  C acc{R(0), R(0)};
  if (r < hi) {
    acc = ldc<R>(&y[r]);
    for (int c = 0; c < wn; ++c) cfms(acc, ldc<R>(&A[(size_t)(n0 + c) * lda + r]), s_x[c]);
    if (blockIdx.x != 0) stc<R>(&y[r], acc);
  }
  if (blockIdx.x != 0) return;
  if (r < hi) s_y[r - b0] = acc;
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  C v0 = lane < wb ? s_y[lane] : C{R(0), R(0)};
  C v1 = lane + 32 < wb ? s_y[lane + 32] : C{R(0), R(0)};
  for (int i = wb - 1; i >= 0; --i) {
    const C src = (i < 32) ? v0 : v1;
    C yi;
    yi.re = __shfl_sync(0xffffffffu, src.re, i & 31);
    yi.im = __shfl_sync(0xffffffffu, src.im, i & 31);
    const C d = s_U[i * NB + i];
    const R den = R(1) / fma(d.re, d.re, d.im * d.im);
    const C xi{(yi.re * d.re + yi.im * d.im) * den, (yi.im * d.re - yi.re * d.im) * den};
    if (lane == i) v0 = xi;
    if (lane + 32 == i) v1 = xi;
    if (lane < i) cfms(v0, s_U[i * NB + lane], xi);
    if (lane + 32 < i) cfms(v1, s_U[i * NB + lane + 32], xi);
  }
  if (lane < wb) stc<R>(&y[b0 + lane], v0);
  if (lane + 32 < wb) stc<R>(&y[b0 + lane + 32], v1);
}

// ---------------------------------------------------------------------------
// k_trsv: the forward and back substitutions with the stored factors in ONE
// cooperative launch.  The CTAs form one group per problem (`group` CTAs
// each); a group walks the forward panels, then the backward 64-row blocks,
// with one bounded group barrier per step.  In every step each CTA of the
// group solves the step's small diagonal triangle redundantly in shared
// memory (warp 0), then updates its share of the remaining rows, rebalanced
// every step (64 rows x 4 column groups per pass).
//
// Forward (panel p, rows [k, k+w)): the panel's row interchanges are replayed
// by gathering from buffer B[p%2] and every updated row is written to
// B[(p+1)%2] (B0 = v, B1 = scratch), so gathers never race with updates.
// The solved panel rows go to v, in a step that does not read v (odd p), or
// one step later (even p).  Backward (U x = y, y in v): rows of the current
// block are read and rows above it are updated in place; the solution
// collects in a second scratch vector that is copied into v at the end.
// ---------------------------------------------------------------------------
struct TrsvArgs {
  const void* A;
  size_t lda, bstride;
  int nn, batch, group, npanels, forward;
  const int* pstart;  // [npanels + 1] first row of each forward panel, then nn
  const int* perm;    // [panel][batch][kPermStride] gather lists
  void* v;            // problem b at v + b * vstride: right-hand side in, solution out
  size_t vstride;
  void* w;            // scratch: [batch][2][nn]
  unsigned* ctr;      // [batch] group barrier counters, zero at launch
  int* status;
};
constexpr int kTrsvBlk = 64;

// dst[r] = src[r] - sum_{c < w} M(r, c0 + c) x_c for rows [lo, hi).  256 threads:
// 64 rows x 4 column groups per pass, partial sums combined in shared memory.
template <typename R>
__device__ __forceinline__ void trsv_rows(const typename Elt<R>::T* __restrict__ A, size_t lda, int c0, int w,
                                          const cpx<R>* s_x, const typename Elt<R>::T* src,
                                          typename Elt<R>::T* dst, int lo, int hi, cpx<R> (*s_part)[64]) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  const int rl = threadIdx.x & 63, cg = threadIdx.x >> 6;
  const int cw = (w + 3) >> 2, cb = cg * cw, ce = min(w, cb + cw);
  for (int base = lo; base < hi; base += 64) {
    const int r = base + rl;
    C part{R(0), R(0)};
    C acc{R(0), R(0)};
    if (r < hi) {
      if (cg == 0) acc = ldc_cg<R>(&src[r]);
      const E* col = A + (size_t)(c0 + cb) * lda + r;
#pragma unroll 16
      for (int c = cb; c < ce; ++c) {
        const E t = __ldg(col);
        col += lda;
        const C xc = s_x[c];
        part.re = fma(t.x, xc.re, fma(-t.y, xc.im, part.re));
        part.im = fma(t.x, xc.im, fma(t.y, xc.re, part.im));
      }
    }
    s_part[cg][rl] = part;
    __syncthreads();
    if (cg == 0 && r < hi) {
      acc.re -= (s_part[0][rl].re + s_part[1][rl].re) + (s_part[2][rl].re + s_part[3][rl].re);
      acc.im -= (s_part[0][rl].im + s_part[1][rl].im) + (s_part[2][rl].im + s_part[3][rl].im);
      stc<R>(&dst[r], acc);
    }
    __syncthreads();
  }
}

// The w x w block at (r0, c0) into s_T (column-major, ld 64): 256 threads as
// 64 rows x 4 groups of 16 columns; all 16 loads of a thread are issued
// before any shared-memory store, so the block costs one memory round trip.
template <typename R>
__device__ __forceinline__ void trsv_load_block(const typename Elt<R>::T* __restrict__ A, size_t lda, int r0, int c0,
                                                int w, cpx<R>* s_T, cpx<R>* s_rdiag = nullptr) {
  using E = typename Elt<R>::T;
  const int r = threadIdx.x & 63, cg = threadIdx.x >> 6;
  E t[16];
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int c = cg * 16 + u;
    if (r < w && c < w) t[u] = __ldg(&A[(size_t)(c0 + c) * lda + r0 + r]);
  }
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int c = cg * 16 + u;
    if (r < w && c < w) s_T[c * kTrsvBlk + r] = cpx<R>{t[u].x, t[u].y};
    if (s_rdiag && r < w && c == r) s_rdiag[r] = crcp(cpx<R>{t[u].x, t[u].y});
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_trsv(TrsvArgs a) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_T = reinterpret_cast<C*>(smem_raw);  // [64][64] diagonal triangle, column-major
  __shared__ C s_g[128];                    // gathered values / right-hand block
  __shared__ C s_x[kTrsvBlk];
  __shared__ C s_xprev[kTrsvBlk];
  __shared__ C s_part[4][64];
  __shared__ C s_rd[kTrsvBlk];  // reciprocals of the diagonal of U (backward)
  const int prob = blockIdx.x / a.group, rank = blockIdx.x % a.group, G = a.group;
  if (prob >= a.batch) return;
  const unsigned long long wlim = wait_limit(a.status);
  const E* A = static_cast<const E*>(a.A) + (size_t)prob * a.bstride;
  E* v = static_cast<E*>(a.v) + (size_t)prob * a.vstride;
  E* b1 = static_cast<E*>(a.w) + (size_t)prob * 2 * a.nn;
  E* xo = b1 + a.nn;
  const int nn = a.nn;
  unsigned* ctr = a.ctr + prob;
  unsigned epoch = 0;

  if (a.forward) {
    int kprev = 0, wprev = 0;
    for (int p = 0; p < a.npanels; ++p) {
      const int k = a.pstart[p], w = a.pstart[p + 1] - k;
      E* cur = (p & 1) ? b1 : v;
      E* nxt = (p & 1) ? v : b1;
      const int* pl = a.perm + ((size_t)p * a.batch + prob) * kPermStride;
      const int count = pl[0];
      for (int e = threadIdx.x; e < count; e += blockDim.x) s_g[e] = ldc_cg<R>(&cur[pl[2 + 2 * e]]);
      trsv_load_block<R>(A, a.lda, k, k, w, s_T);
      __syncthreads();
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        C v0 = lane < w ? s_g[lane] : C{R(0), R(0)};
        C v1 = lane + 32 < w ? s_g[lane + 32] : C{R(0), R(0)};
        for (int i = 0; i < w; ++i) {
          const C src = (i < 32) ? v0 : v1;
          C ui;
          ui.re = __shfl_sync(0xffffffffu, src.re, i & 31);
          ui.im = __shfl_sync(0xffffffffu, src.im, i & 31);
          if (lane > i && lane < w) cfms(v0, s_T[i * kTrsvBlk + lane], ui);
          if (lane + 32 > i && lane + 32 < w) cfms(v1, s_T[i * kTrsvBlk + lane + 32], ui);
        }
        if (lane < w) s_x[lane] = v0;
        if (lane + 32 < w) s_x[lane + 32] = v1;
      }
      __syncthreads();
      if (rank == 0 && (p & 1)) {  // v is not read in odd steps
        for (int i = threadIdx.x; i < wprev; i += blockDim.x) stc<R>(&v[kprev + i], s_xprev[i]);
        for (int i = threadIdx.x; i < w; i += blockDim.x) stc<R>(&v[k + i], s_x[i]);
      }
      const int r0 = k + w;
      if (r0 < nn) {
        const int per = (nn - r0 + G - 1) / G;
        const int lo = min(nn, r0 + rank * per), hi = min(nn, lo + per);
        trsv_rows<R>(A, a.lda, k, w, s_x, cur, nxt, lo, hi, s_part);
        // rows that received a displaced panel row start from the gathered value
        for (int e = w + threadIdx.x; e < count; e += blockDim.x) {
          const int r = pl[1 + 2 * e];
          if (r >= lo && r < hi) {
            C acc = s_g[e];
            const E* row = A + (size_t)k * a.lda + r;
            for (int cb = 0; cb < w; cb += 16) {
              E t[16];
#pragma unroll
              for (int u = 0; u < 16; ++u)
                if (cb + u < w) t[u] = __ldg(row + (size_t)(cb + u) * a.lda);
#pragma unroll
              for (int u = 0; u < 16; ++u)
                if (cb + u < w) cfms(acc, C{t[u].x, t[u].y}, s_x[cb + u]);
            }
            stc<R>(&nxt[r], acc);
          }
        }
      }
      if (p & 1) {
        wprev = 0;
      } else {
        for (int i = threadIdx.x; i < w; i += blockDim.x) s_xprev[i] = s_x[i];
        kprev = k;
        wprev = w;
      }
      if (!grid_barrier(ctr, ++epoch, G, a.status, wlim)) return;
    }
    if (wprev > 0) {  // the last panel was even: its rows still go to v
      if (rank == 0)
        for (int i = threadIdx.x; i < wprev; i += blockDim.x) stc<R>(&v[kprev + i], s_xprev[i]);
      if (!grid_barrier(ctr, ++epoch, G, a.status, wlim)) return;
    }
  }

  const int nblk = (nn + kTrsvBlk - 1) / kTrsvBlk;
  for (int sb = nblk - 1; sb >= 0; --sb) {
    const int b0 = sb * kTrsvBlk, wb = min(kTrsvBlk, nn - b0);
    for (int i = threadIdx.x; i < wb; i += blockDim.x) s_g[i] = ldc_cg<R>(&v[b0 + i]);
    trsv_load_block<R>(A, a.lda, b0, b0, wb, s_T, s_rd);
    __syncthreads();
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      C v0 = lane < wb ? s_g[lane] : C{R(0), R(0)};
      C v1 = lane + 32 < wb ? s_g[lane + 32] : C{R(0), R(0)};
      for (int i = wb - 1; i >= 0; --i) {
        const C src = (i < 32) ? v0 : v1;
        C yi;
        yi.re = __shfl_sync(0xffffffffu, src.re, i & 31);
        yi.im = __shfl_sync(0xffffffffu, src.im, i & 31);
        const C xi = yi * s_rd[i];
        if (lane == i) v0 = xi;
        if (lane + 32 == i) v1 = xi;
        if (lane < i) cfms(v0, s_T[i * kTrsvBlk + lane], xi);
        if (lane + 32 < i) cfms(v1, s_T[i * kTrsvBlk + lane + 32], xi);
      }
      if (lane < wb) s_x[lane] = v0;
      if (lane + 32 < wb) s_x[lane + 32] = v1;
    }
    __syncthreads();
    if (rank == 0)
      for (int i = threadIdx.x; i < wb; i += blockDim.x) stc<R>(&xo[b0 + i], s_x[i]);
    if (b0 > 0) {
      const int per = (b0 + G - 1) / G;
      const int lo = min(b0, rank * per), hi = min(b0, lo + per);
      trsv_rows<R>(A, a.lda, b0, wb, s_x, v, v, lo, hi, s_part);
    }
    if (!grid_barrier(ctr, ++epoch, G, a.status, wlim)) return;
  }
  const int per = (nn + G - 1) / G;
  const int lo = min(nn, rank * per), hi = min(nn, lo + per);
  for (int r = lo + threadIdx.x; r < hi; r += blockDim.x) v[r] = __ldcg(&xo[r]);
}

// ---------------------------------------------------------------------------
// FP32 solves (the mixed form's refinement) with inverted diagonal blocks.
// k_tri_inv inverts, once per factorisation, every diagonal block the solves
// step through: blocks [0, npanels) are the unit-lower L11 of the forward
// panels (w x w at (k, k)), blocks [npanels, npanels + nblk) the upper
// triangles of the 64-row backward blocks.  Thread j solves T x = e_j; the
// inverse is stored row-major [64][64], zero outside the block.  The factors
// come from partial pivoting (|L| <= 1), and the FP32 solves only
// precondition the FP64 refinement, so explicit block inverses are accurate
// enough there; the FP64 solves keep the substitution of k_trsv.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(64) k_tri_inv(const float2* __restrict__ Abase, size_t lda, size_t bstride, int nn,
                                                int npanels, const int* __restrict__ pstart, float2* inv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto s_T = reinterpret_cast<zf(*)[65]>(smem_raw);  // [64][65]: [column][row]
  auto s_X = s_T + 64;                                // [64][65]: [column j of the inverse][row]
  const int b = blockIdx.x, prob = blockIdx.y, j = threadIdx.x;
  const int nblk = (nn + kTrsvBlk - 1) / kTrsvBlk;
  const float2* A = Abase + (size_t)prob * bstride;
  float2* out = inv + ((size_t)prob * (npanels + nblk) + b) * kTrsvBlk * kTrsvBlk;
  const bool lower = b < npanels;
  const int k0 = lower ? pstart[b] : (b - npanels) * kTrsvBlk;
  const int w = lower ? pstart[b + 1] - k0 : min(kTrsvBlk, nn - k0);
  for (int c = 0; c < w; ++c)
    if (j < w) {
      const float2 t = A[(size_t)(k0 + c) * lda + k0 + j];
      s_T[c][j] = zf{t.x, t.y};
    }
  __syncthreads();
  if (j < w) {
    if (lower) {  // x_i = [i == j] - sum_{j <= k < i} L(i,k) x_k
      for (int i = 0; i < j; ++i) s_X[j][i] = zf{0.f, 0.f};
      s_X[j][j] = zf{1.f, 0.f};
      for (int i = j + 1; i < w; ++i) {
        zf acc{0.f, 0.f};
        for (int kk = j; kk < i; ++kk) cfms(acc, s_T[kk][i], s_X[j][kk]);
        s_X[j][i] = acc;
      }
    } else {  // x_i = ([i == j] - sum_{i < k <= j} U(i,k) x_k) / U(i,i)
      for (int i = j + 1; i < w; ++i) s_X[j][i] = zf{0.f, 0.f};
      for (int i = j; i >= 0; --i) {
        zf acc{i == j ? 1.f : 0.f, 0.f};
        for (int kk = i + 1; kk <= j; ++kk) cfms(acc, s_T[kk][i], s_X[j][kk]);
        const zf d = s_T[i][i];
        s_X[j][i] = (d.re == 0.f && d.im == 0.f) ? zf{0.f, 0.f} : acc * crcp(d);
      }
    }
  }
  __syncthreads();
  for (int i = 0; i < kTrsvBlk; ++i) {
    const zf x = (i < w && j < w) ? s_X[j][i] : zf{0.f, 0.f};
    out[(size_t)i * kTrsvBlk + j] = make_float2(x.re, x.im);
  }
}

__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_rows_load(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_rows_prefetch(const CUtensorMap* map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(map), "r"(x), "r"(y),
               "r"(z)
               : "memory");
}

// k_trsv with the FP32 factors, same group structure, gathers and buffers
// (see k_trsv), three changes per step: (1) the step's diagonal triangle is
// applied as its precomputed inverse (a 64 x 64 product over 256 threads
// instead of a 64-step warp solve); (2) this CTA's share of the step's L (or
// U) rows is brought into shared memory by one TMA box load issued when the
// step starts, before the gather and the product it does not depend on; (3)
// the next step's rows and inverse are prefetched into L2 meanwhile.  A box
// is `ldl` rows (even, <= 256) by 64 columns of the rows map `tm` (8-byte
// elements; rows past nn read as zero); 1, 2 or 4 threads per row for the
// row updates.
__global__ void __launch_bounds__(256) k_trsv_f32(const __grid_constant__ CUtensorMap tm, TrsvArgs a,
                                                  const float2* __restrict__ tinv, int ldl, int ninv_l) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // [64][ldl] this CTA's rows of the step's columns: a TMA tile destination,
  // so 128-byte aligned (the launch adds 128 bytes for the rounding)
  float2* s_L = reinterpret_cast<float2*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
  int* s_ovr = reinterpret_cast<int*>(s_L + (size_t)kTrsvBlk * ldl);  // [ldl] gather entry of a displaced row, or -1
  __shared__ zf s_g[128];
  __shared__ zf s_x[kTrsvBlk];
  __shared__ zf s_xprev[kTrsvBlk];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ int s_pl[kPermStride];  // the step's gather list: count, then dst/src pairs
  __shared__ int s_ok;
  const int prob = blockIdx.x / a.group, rank = blockIdx.x % a.group, G = a.group;
  if (prob >= a.batch) return;
  const unsigned long long wlim = wait_limit(a.status);
  float2* v = static_cast<float2*>(a.v) + (size_t)prob * a.vstride;
  float2* b1 = static_cast<float2*>(a.w) + (size_t)prob * 2 * a.nn;
  float2* xo = b1 + a.nn;
  const int nn = a.nn, tid = threadIdx.x;
  const int nblk = (nn + kTrsvBlk - 1) / kTrsvBlk;
  // inverses of this problem: ninv_l forward panels (of the factorisation), then nblk blocks
  const float2* inv = tinv + (size_t)prob * (ninv_l + nblk) * kTrsvBlk * kTrsvBlk;
  unsigned* ctr = a.ctr + prob;
  unsigned epoch = 0, phase = 0;
  if (tid == 0) mbar_init(&s_bar, 1);
  for (int i = tid; i < ldl; i += blockDim.x) s_ovr[i] = -1;
  __syncthreads();

  // This CTA's rows of a step whose updated rows are [r0, r1): [lo, hi).
  auto share = [&](int r0, int r1, int& lo, int& hi) {
    const int per = (r1 - r0 + G - 1) / G;
    lo = min(r1, r0 + rank * per);
    hi = min(r1, lo + per);
  };
  // Rows [lo, hi) of columns [c0, c0 + 64) into s_L as one box starting
  // at the even row below lo (16-byte aligned), or its L2 prefetch.
  auto fetch = [&](int c0, int lo, int hi, bool prefetch) {
    if (prefetch) {
      if (hi > lo) tma_rows_prefetch(&tm, lo & ~1, c0, prob);
      return;
    }
    mbar_expect_tx(&s_bar, hi > lo ? (unsigned)ldl * kTrsvBlk * 8u : 0u);
    if (hi > lo) tma_rows_load(s_L, &tm, lo & ~1, c0, prob, &s_bar);
  };
  // dst[r] = base[r] - sum_{c < w} s_L[c][r - la] x_c for rows [lo, hi),
  // base = the gathered value of a displaced row (s_ovr) or src[r]; tpr
  // threads per row (consecutive lanes) combine their columns by shuffles.
  auto update_rows = [&](int lo, int hi, int w, const float2* src, float2* dst) {
    const int rows = hi - lo, la = lo & ~1;
    const int tpr = rows <= 64 ? 4 : (rows <= 128 ? 2 : 1), rpp = 256 / tpr;
    const int sub = tid & (tpr - 1), rl = tid / tpr;
    const int passes = (rows + rpp - 1) / rpp;
    for (int ps = 0; ps < passes; ++ps) {
      const int r = lo + ps * rpp + rl;
      const bool act = r < hi;
      // the base value first: its load overlaps the products below
      const int e = act && sub == 0 ? s_ovr[r - lo] : -1;
      zf base{0.f, 0.f};
      if (act && sub == 0) base = e >= 0 ? s_g[e] : ldc_cg<float>(&src[r]);
      zf acc{0.f, 0.f}, acc2{0.f, 0.f};
      if (act) {
        const float2* col = s_L + (r - la);
        for (int c = sub; c < w; c += 2 * tpr) {
          const float2 t0 = col[(size_t)c * ldl];
          cfms(acc, zf{t0.x, t0.y}, s_x[c]);
          if (c + tpr < w) {
            const float2 t1 = col[(size_t)(c + tpr) * ldl];
            cfms(acc2, zf{t1.x, t1.y}, s_x[c + tpr]);
          }
        }
      }
      acc.re += acc2.re;
      acc.im += acc2.im;
      for (int off = 1; off < tpr; off <<= 1) {
        acc.re += __shfl_xor_sync(0xffffffffu, acc.re, off);
        acc.im += __shfl_xor_sync(0xffffffffu, acc.im, off);
      }
      if (act && sub == 0) {
        if (e >= 0) s_ovr[r - lo] = -1;
        stc<float>(&dst[r], zf{base.re + acc.re, base.im + acc.im});
      }
    }
  };
  // x = inv(block) g for the step's w values: 4 threads per row, 16 columns
  // each; the thread's 16 inverse entries are loaded first (load_inv, at the
  // start of the step: they do not depend on g).
  float4 tv[8];
  auto load_inv = [&](const float2* blk) {
    const float4* row = reinterpret_cast<const float4*>(blk + (size_t)(tid >> 2) * kTrsvBlk + 16 * (tid & 3));
#pragma unroll
    for (int u = 0; u < 8; ++u) tv[u] = __ldg(row + u);
  };
  auto apply_inv = [&](int w) {
    const int i = tid >> 2, q = tid & 3;
    zf acc{0.f, 0.f};
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const float4 t = tv[u];
      const int jj = 16 * q + 2 * u;
      if (jj < w) cfms(acc, zf{-t.x, -t.y}, s_g[jj]);
      if (jj + 1 < w) cfms(acc, zf{-t.z, -t.w}, s_g[jj + 1]);
    }
#pragma unroll
    for (int off = 1; off < 4; off <<= 1) {
      acc.re += __shfl_xor_sync(0xffffffffu, acc.re, off);
      acc.im += __shfl_xor_sync(0xffffffffu, acc.im, off);
    }
    if (q == 0 && i < w) s_x[i] = acc;
  };

  // The steps: forward panels s < nf, then backward blocks.  Step s works
  // on columns [c0, c0 + w) (inverse block ib) and updates rows [r0, r1).
  const int nf = a.forward ? a.npanels : 0, nsteps = nf + nblk;
  auto desc = [&](int st, int& c0, int& w, int& r0, int& r1, int& ib) {
    if (st < nf) {
      c0 = __ldg(&a.pstart[st]);
      w = __ldg(&a.pstart[st + 1]) - c0;
      r0 = c0 + w;
      r1 = nn;
      ib = st;
    } else {
      const int sb = nblk - 1 - (st - nf);
      c0 = sb * kTrsvBlk;
      w = min(kTrsvBlk, nn - c0);
      r0 = 0;
      r1 = c0;
      ib = ninv_l + sb;
    }
  };
  // The loads of step st that do not depend on the previous step's values:
  // this CTA's rows (TMA box), its inverse entries (registers), the panel's
  // gather list (shared memory), and the L2 prefetch of step st + 1.
  auto issue = [&](int st) {
    int c0, w, r0, r1, ib, lo, hi;
    desc(st, c0, w, r0, r1, ib);
    share(r0, r1, lo, hi);
    if (tid == 0) {
      fetch(c0, lo, hi, false);
      if (st + 1 < nsteps) {
        int c1, w1, q0, q1, ib1, lo1, hi1;
        desc(st + 1, c1, w1, q0, q1, ib1);
        share(q0, q1, lo1, hi1);
        fetch(c1, lo1, hi1, true);
        bulk_prefetch_l2(inv + (size_t)ib1 * kTrsvBlk * kTrsvBlk, kTrsvBlk * kTrsvBlk * 8u);
      }
    }
    load_inv(inv + (size_t)ib * kTrsvBlk * kTrsvBlk);
    if (st < nf) {
      const int* pl = a.perm + ((size_t)st * a.batch + prob) * kPermStride;
      for (int i = tid; i < kPermStride; i += blockDim.x) s_pl[i] = __ldg(&pl[i]);
    }
  };

  int kprev = 0, wprev = 0;
  issue(0);
  __syncthreads();
  for (int st = 0; st < nsteps; ++st) {
    int c0, w, r0, r1, ib, lo, hi;
    desc(st, c0, w, r0, r1, ib);
    share(r0, r1, lo, hi);
    const bool fwd = st < nf, odd = st & 1;
    float2* cur = fwd ? (odd ? b1 : v) : v;
    float2* nxt = fwd ? (odd ? v : b1) : v;
    if (fwd) {  // the panel's interchanges, replayed as a gather
      const int count = s_pl[0];
      for (int e = tid; e < count; e += blockDim.x) {
        s_g[e] = ldc_cg<float>(&cur[s_pl[2 + 2 * e]]);
        const int r = s_pl[1 + 2 * e];
        if (e >= w && r >= lo && r < hi) s_ovr[r - lo] = e;
      }
    } else {
      for (int i = tid; i < w; i += blockDim.x) s_g[i] = ldc_cg<float>(&v[c0 + i]);
    }
    __syncthreads();
    apply_inv(w);  // s_x = L11^-1 (gathered panel rows) or U_bb^-1 y_b
    __syncthreads();
    if (fwd && rank == 0 && odd) {  // v is not read in odd forward steps
      for (int i = tid; i < wprev; i += blockDim.x) stc<float>(&v[kprev + i], s_xprev[i]);
      for (int i = tid; i < w; i += blockDim.x) stc<float>(&v[c0 + i], s_x[i]);
    }
    if (!fwd && rank == 0)
      for (int i = tid; i < w; i += blockDim.x) stc<float>(&xo[c0 + i], s_x[i]);
    if (!mbar_wait(&s_bar, phase, wlim)) {
      atomicExch(&a.status[ST_TIMEOUT], 1);
      mbar_wait(&s_bar, phase, wlim);  // let the box in flight land before leaving
      return;
    }
    phase ^= 1u;
    // rows [lo, hi): nxt = cur - L x (a row that received a displaced panel
    // row starts from the gathered value), or v -= U x in place
    update_rows(lo, hi, w, cur, nxt);
    if (fwd) {
      if (odd) {
        wprev = 0;
      } else {
        for (int i = tid; i < w; i += blockDim.x) s_xprev[i] = s_x[i];
        kprev = c0;
        wprev = w;
      }
    }
    // Group barrier, split: arrive, issue the next step's loads, then wait.
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      red_release_gpu_add(ctr, 1u);
    }
    ++epoch;
    if (st + 1 < nsteps) issue(st + 1);
    if (tid == 0) {
      const unsigned target = epoch * (unsigned)G;
      const unsigned long long t0 = globaltimer_ns();
      int ok = 1;
      unsigned spins = 0;
      while (ld_acquire_gpu(ctr) < target) {
        if ((++spins & 255u) == 0) {
          if (*(volatile int*)&a.status[ST_TIMEOUT] != 0 || globaltimer_ns() - t0 > wlim) {
            atomicExch(&a.status[ST_TIMEOUT], 1);
            ok = 0;
            break;
          }
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    if (!s_ok) {
      if (st + 1 < nsteps) mbar_wait(&s_bar, phase, wlim);  // the next step's box, issued above, lands first
      return;
    }
    if (st == nf - 1 && wprev > 0) {  // the last panel was even: its rows still go to v
      if (rank == 0)
        for (int i = tid; i < wprev; i += blockDim.x) stc<float>(&v[kprev + i], s_xprev[i]);
      if (!grid_barrier(ctr, ++epoch, G, a.status, wlim)) {
        if (st + 1 < nsteps) mbar_wait(&s_bar, phase, wlim);  // the next step's box lands first
        return;
      }
    }
  }
  int lo, hi;
  share(0, nn, lo, hi);
  for (int r = lo + tid; r < hi; r += blockDim.x) v[r] = __ldcg(&xo[r]);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
int lu_ensure_workspace(bem_ctx* ctx, int nn, int batch) {
  LuWork& L = ctx->lu;
  if (L.cap_nn >= nn && L.cap_batch >= batch && L.ipiv) return BEM_OK;
  dev_free(ctx, L.ipiv);
  dev_free(ctx, L.perm);
  L.ipiv = nullptr;
  L.perm = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &L.ipiv, (size_t)nn * batch * sizeof(int)));
  const int max_panels = (nn + 15) / 16 + 1;
  BEM_CUDA(ctx, dev_alloc(ctx, &L.perm, (size_t)max_panels * kPermStride * batch * sizeof(int)));
  dev_free(ctx, L.pstart);
  L.pstart = nullptr;
  BEM_CUDA(ctx, dev_alloc(ctx, &L.pstart, (size_t)(max_panels + 1) * sizeof(int)));
  L.cap_nn = nn;
  L.cap_batch = batch;
  if (!L.slot_val) {
    BEM_CUDA(ctx, dev_alloc(ctx, &L.slot_val, 2 * kMaxGrid * sizeof(double)));
    BEM_CUDA(ctx, dev_alloc(ctx, &L.slot_row, 2 * kMaxGrid * sizeof(int)));
    BEM_CUDA(ctx, dev_alloc(ctx, &L.cand, (size_t)2 * kMaxGrid * 64 * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &L.drow, 2 * 64 * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &L.barrier, sizeof(unsigned)));
  }
  return BEM_OK;
}

constexpr size_t kPanelSmemBudget = 220 * 1024;

template <typename R, int NB>
static size_t push_panel_smem(int rp) {
  return ((size_t)NB * rp + (size_t)kPushMoves * NB) * sizeof(cpx<R>);
}

template <typename R, int NB, int NT>
static int launch_cluster_panel(bem_ctx* ctx, const PanelArgs& pa, int batch) {
  const bool push = ctx->panel_push;
  const size_t smem = push ? push_panel_smem<R, NB>(pa.rp) : ((size_t)NB * pa.rp + 4 * NB + 2 * 8 * NB) * sizeof(cpx<R>);
  auto kern = push ? k_panel_push<R, NB, NT> : k_panel_cluster<R, NB, NT>;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(kern), smem));
  BEM_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pa.cs, batch, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pa.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BEM_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, pa));
  return BEM_OK;
}

// Does a panel of width NB with rp rows per CTA fit one CTA's shared memory?
template <typename R, int NB, int NT>
static bool cluster_panel_fits(int rp) {
  // both forms (pull and push) must fit, so that either can run any panel
  cudaFuncAttributes fa{}, fp{};
  if (cudaFuncGetAttributes(&fa, k_panel_cluster<R, NB, NT>) != cudaSuccess) return false;
  if (cudaFuncGetAttributes(&fp, k_panel_push<R, NB, NT>) != cudaSuccess) return false;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t dyn = ((size_t)NB * rp + 4 * NB + 2 * 8 * NB) * sizeof(cpx<R>);
  return dyn + fa.sharedSizeBytes + 1024 <= (size_t)optin &&
         push_panel_smem<R, NB>(rp) + fp.sharedSizeBytes + 1024 <= (size_t)optin;
}

template <typename R>
static bool cluster_panel_fits_any(int nb, int rp) {
  const bool big = rp > 256;
  if (nb == 64) return big ? cluster_panel_fits<R, 64, 512>(rp) : cluster_panel_fits<R, 64, 256>(rp);
  if (nb == 32) return big ? cluster_panel_fits<R, 32, 512>(rp) : cluster_panel_fits<R, 32, 256>(rp);
  if (nb == 16) return big ? cluster_panel_fits<R, 16, 512>(rp) : cluster_panel_fits<R, 16, 256>(rp);
  return false;
}

template <int NB>
static size_t calu_dyn_smem(int rp) {
  return ((size_t)NB * rp + (size_t)std::max(kCaluCand * kCaluSW, kCaluMoves * NB)) * sizeof(zf);
}

template <int NB, int NT>
static bool calu_panel_fits(int rp) {
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, k_panel_calu<NB, NT>) != cudaSuccess) return false;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return calu_dyn_smem<NB>(rp) + fa.sharedSizeBytes + 1024 <= (size_t)optin;
}

static bool calu_panel_fits_any(int nb, int rp) {
  const bool big = rp > 256;
  if (nb == 64) return big ? calu_panel_fits<64, 512>(rp) : calu_panel_fits<64, 256>(rp);
  if (nb == 32) return big ? calu_panel_fits<32, 512>(rp) : calu_panel_fits<32, 256>(rp);
  if (nb == 16) return big ? calu_panel_fits<16, 512>(rp) : calu_panel_fits<16, 256>(rp);
  return false;
}

template <int NB, int NT>
static int launch_calu_panel(bem_ctx* ctx, const PanelArgs& pa, int batch) {
  const size_t smem = calu_dyn_smem<NB>(pa.rp);
  auto kern = k_panel_calu<NB, NT>;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(kern), smem));
  BEM_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(pa.cs, batch, 1);
  cfg.blockDim = dim3(NT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = pa.cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  BEM_CUDA(ctx, cudaLaunchKernelEx(&cfg, kern, pa));
  return BEM_OK;
}

static int launch_calu_panel_any(bem_ctx* ctx, const PanelArgs& pa, int batch, int nb) {
  const bool big = pa.rp > 256;
  if (nb == 64) return big ? launch_calu_panel<64, 512>(ctx, pa, batch) : launch_calu_panel<64, 256>(ctx, pa, batch);
  if (nb == 32) return big ? launch_calu_panel<32, 512>(ctx, pa, batch) : launch_calu_panel<32, 256>(ctx, pa, batch);
  if (nb == 16) return big ? launch_calu_panel<16, 512>(ctx, pa, batch) : launch_calu_panel<16, 256>(ctx, pa, batch);
  return fail(ctx, BEM_ERR_ARG, "no tournament panel variant for this size");
}

// Dispatch on (panel width, threads = rows per CTA rounded up to 256 or 512).
template <typename R>
static int launch_cluster_panel_any(bem_ctx* ctx, const PanelArgs& pa, int batch, int nb) {
  const bool big = pa.rp > 256;
  if (nb == 64) return big ? launch_cluster_panel<R, 64, 512>(ctx, pa, batch) : launch_cluster_panel<R, 64, 256>(ctx, pa, batch);
  if (nb == 32) return big ? launch_cluster_panel<R, 32, 512>(ctx, pa, batch) : launch_cluster_panel<R, 32, 256>(ctx, pa, batch);
  if (nb == 16) return big ? launch_cluster_panel<R, 16, 512>(ctx, pa, batch) : launch_cluster_panel<R, 16, 256>(ctx, pa, batch);
  return fail(ctx, BEM_ERR_ARG, "no cluster panel variant for this size");
}

template <typename R, int NB>
static int launch_grid_panel(bem_ctx* ctx, PanelArgs pa) {
  auto kern = k_panel_grid<R, NB>;
  const size_t smem = (size_t)pa.rp * NB * sizeof(cpx<R>);
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(kern), smem));
  BEM_CUDA(ctx, cudaMemsetAsync(pa.bar, 0, sizeof(unsigned), ctx->stream));
  void* args[] = {&pa};
  BEM_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)kern, dim3(pa.cs), dim3(kPanelThreads), args, smem,
                                            ctx->stream));
  return BEM_OK;
}

// Largest cluster size the device accepts for the panel kernel (16, else 8).
static int cluster_size(bem_ctx* ctx) {
  if (ctx->lu.cluster_cs) return ctx->lu.cluster_cs;
  int cs = 8;
  auto kern = k_panel_cluster<double, 32, 512>;
  raise_smem_limit(reinterpret_cast<const void*>(kern), kPanelSmemBudget);
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(512, 1, 1);
    cfg.dynamicSmemBytes = kPanelSmemBudget;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) == cudaSuccess && nclusters >= 1) cs = 16;
  }
  cudaGetLastError();
  ctx->lu.cluster_cs = cs;
  return cs;
}

// CTAs per panel cluster for an nn x nn system: the device's largest (16)
// halved while every CTA still holds at most 256 panel rows (option
// "small_clusters", on).  A panel costs about the same time per column
// whatever the cluster size, so small systems need no more than a few CTAs
// each, and the lockstep batches and concurrent classes of small problems
// then fit many more problems on the device at once.  The 6480-unknown
// sweep keeps 16.
static int cluster_size_for(bem_ctx* ctx, int nn) {
  int cs = cluster_size(ctx);
  if (ctx->small_clusters)
    while (cs > 2 && (nn + cs / 2 - 1) / (cs / 2) <= 256) cs /= 2;
  return cs;
}

// Clusters of the panel kernel that can be resident at once (0 if unknown).
template <typename R, int NB, int NT>
static int cluster_capacity(int cs, int rp) {
  const size_t smem = ((size_t)NB * rp + 4 * NB + 2 * 8 * NB) * sizeof(cpx<R>);
  auto kern = k_panel_cluster<R, NB, NT>;
  int n = 0;
  if (raise_smem_limit(reinterpret_cast<const void*>(kern), smem) == cudaSuccess &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) n = 0;
  }
  cudaGetLastError();
  return n;
}

template <typename R>
static int lockstep_capacity_t(bem_ctx* ctx, int nn) {
  const int cs = cluster_size_for(ctx, nn);
  const int rp = (nn + cs - 1) / cs;
  if (rp > 512) return kMaxBatch;  // grid-panel fallback: problems take turns anyway
  const bool big = rp > 256;
  for (int nb : {64, 32, 16}) {
    if (!cluster_panel_fits_any<R>(nb, rp)) continue;
    int n = 0;
    if (nb == 64) n = big ? cluster_capacity<R, 64, 512>(cs, rp) : cluster_capacity<R, 64, 256>(cs, rp);
    if (nb == 32) n = big ? cluster_capacity<R, 32, 512>(cs, rp) : cluster_capacity<R, 32, 256>(cs, rp);
    if (nb == 16) n = big ? cluster_capacity<R, 16, 512>(cs, rp) : cluster_capacity<R, 16, 256>(cs, rp);
    // At most one CTA per SM: clusters that share SMs (the occupancy query
    // allows two CTAs per SM for short panels) measured 2.75x the time of a
    // one-per-SM launch, where two launches of half the problems take 2x.
    const int one_per_sm = std::max(1, ctx->num_sms / cs);
    return n >= 1 ? std::min({n, one_per_sm, kMaxBatch}) : std::min(one_per_sm, kMaxBatch);
  }
  return kMaxBatch;
}

// FP64 trailing update by cuBLAS (option f64_cublas): C -= L U for rows
// [r0, nn) and columns [c0, cend) of `batch` systems, one strided-batched
// ZGEMM (the plain library GEMM, FP64 tensor cores).  L is A's columns
// kcol..kcol+kw-1 at rows r0.., or `lg` (ld nn - r0, lg_stride per problem);
// U is A's rows kcol..kcol+kw-1 at columns c0...  The handle and a fixed
// workspace are made once per context, so a captured graph allocates nothing.
constexpr size_t kCublasWorkspace = (size_t)32 << 20;

int f64_gemm_cublas(bem_ctx* ctx, double2* A, size_t lda, size_t bstride, int nn, int kcol, int kw, int r0, int c0,
                    int cend, int batch, const double2* lg, size_t lg_stride) {
  if (!ctx->cublas) {
    cublasHandle_t h = nullptr;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return fail(ctx, BEM_ERR_CUDA, "cublasCreate failed");
    ctx->cublas = h;
    BEM_CUDA(ctx, dev_alloc(ctx, reinterpret_cast<unsigned char**>(&ctx->cublas_ws), kCublasWorkspace));
    BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (cublasSetWorkspace(h, ctx->cublas_ws, kCublasWorkspace) != CUBLAS_STATUS_SUCCESS)
      return fail(ctx, BEM_ERR_CUDA, "cublasSetWorkspace failed");
  }
  cublasHandle_t h = static_cast<cublasHandle_t>(ctx->cublas);
  if (cublasSetStream(h, ctx->stream) != CUBLAS_STATUS_SUCCESS) return fail(ctx, BEM_ERR_CUDA, "cublasSetStream failed");
  const int m = nn - r0, n = cend - c0;
  if (m <= 0 || n <= 0 || kw <= 0) return BEM_OK;
  const cuDoubleComplex minus_one = make_cuDoubleComplex(-1.0, 0.0), one = make_cuDoubleComplex(1.0, 0.0);
  cuDoubleComplex* a = reinterpret_cast<cuDoubleComplex*>(A);
  const cuDoubleComplex* l = lg ? reinterpret_cast<const cuDoubleComplex*>(lg) : a + (size_t)kcol * lda + r0;
  const int ldl = lg ? m : (int)lda;
  const long long sl = lg ? (long long)lg_stride : (long long)bstride;
  const cublasStatus_t st = cublasZgemmStridedBatched(
      h, CUBLAS_OP_N, CUBLAS_OP_N, m, n, kw, &minus_one, l, ldl, sl, a + (size_t)c0 * lda + kcol, (int)lda,
      (long long)bstride, &one, a + (size_t)c0 * lda + r0, (int)lda, (long long)bstride, batch);
  if (st != CUBLAS_STATUS_SUCCESS) return fail(ctx, BEM_ERR_CUDA, "cublasZgemmStridedBatched failed");
  ctx->launches++;
  return BEM_OK;
}

int f64_update_cublas(bem_ctx* ctx, double2* A, size_t lda, size_t bstride, int nn, int k, int w, int c0, int ncols,
                      int batch) {
  return f64_gemm_cublas(ctx, A, lda, bstride, nn, k, w, c0, c0, ncols, batch, nullptr, 0);
}

// L of an FP64 panel pair for its update past the pair (rows r0.. of columns
// k..k+w1+w2-1): the first panel's columns read through the second panel's
// gather list (count, then dst/src pairs; row dst of C takes L from row src,
// as k_gemm_f64 with gperm does), the second panel's as they are.  Out:
// column-major, ld nn - r0, problem b at out + b * ostride.
__global__ void __launch_bounds__(256) k_gather_l_pair(const double2* __restrict__ Abase, size_t lda, size_t bstride,
                                                       int nn, int k, int w1, int w2, int r0,
                                                       const int* __restrict__ gperm, int gperm_stride,
                                                       double2* __restrict__ out, size_t ostride) {
  __shared__ int s_map[256];
  const int b = blockIdx.y, tid = threadIdx.x;
  const int row0 = r0 + blockIdx.x * 256, r = row0 + tid;
  const double2* A = Abase + (size_t)b * bstride;
  double2* o = out + (size_t)b * ostride;
  const int m = nn - r0;
  s_map[tid] = r;
  __syncthreads();
  const int* pl = gperm + (size_t)b * gperm_stride;
  const int cnt = pl[0];
  for (int e = tid; e < cnt; e += blockDim.x) {
    const int dst = pl[1 + 2 * e];
    if (dst >= row0 && dst < row0 + 256) s_map[dst - row0] = pl[2 + 2 * e];
  }
  __syncthreads();
  if (r >= nn) return;
  const int src = s_map[tid];
  for (int c = 0; c < w1 + w2; ++c) o[(size_t)c * m + (r - r0)] = A[(size_t)(k + c) * lda + (c < w1 ? src : r)];
}

void release_cublas(bem_ctx* ctx) {
  if (ctx->cublas) cublasDestroy(static_cast<cublasHandle_t>(ctx->cublas));
  ctx->cublas = nullptr;
  dev_free(ctx, ctx->cublas_ws);
  ctx->cublas_ws = nullptr;
}

// Problems whose panels run in one wave: the first (tallest) panel's cluster
// kernel, as many clusters as can be resident at once.
int lu_lockstep_capacity(bem_ctx* ctx, int nn, bool fp32) {
  // occupancy queries are host calls of tens of microseconds: remember each answer
  const long long key = 4LL * nn + (fp32 ? 1 : 0) + (ctx->small_clusters ? 2 : 0);
  auto it = ctx->lockstep_cache.find(key);
  if (it != ctx->lockstep_cache.end()) return it->second;
  const int cap = fp32 ? lockstep_capacity_t<float>(ctx, nn) : lockstep_capacity_t<double>(ctx, nn);
  ctx->lockstep_cache[key] = cap;
  return cap;
}

template <typename T>
static int ts_ensure(bem_ctx* ctx, T*& p, size_t& cap, size_t need) {
  if (p && cap >= need) return BEM_OK;
  dev_free(ctx, p);
  p = nullptr;
  cap = 0;
  BEM_CUDA(ctx, dev_alloc(ctx, &p, need * sizeof(T)));
  cap = need;
  return BEM_OK;
}

// The 64-column FP32 panel at column k of `batch` problems, taller than one
// cluster holds, by tournament pivoting (the kernels k_tslu_*): its factors go
// into A, its pivots into ipiv, its gather list to perm_p and its start to
// the panel starts (index pidx), as the cluster kernels leave them.
static int tslu_panel(bem_ctx* ctx, float2* A, size_t lda, size_t bstride, int nn, int k, int batch, int* perm_p,
                      int pidx) {
  LuWork& L = ctx->lu;
  const int m = nn - k;
  // as few chunks as let one cluster hold a chunk's 64 columns
  const int cs1 = cluster_size(ctx);
  int nch = 1, chunk = 0;
  for (;; ++nch) {
    chunk = ((m + nch - 1) / nch + 15) & ~15;
    const int rp = (chunk + cs1 - 1) / cs1;
    if (rp <= 512 && cluster_panel_fits_any<float>(kTsluW, rp)) break;
    if (nch >= 64) return fail(ctx, BEM_ERR_ARG, "panel too tall for the tournament");
  }
  const int ncand = nch * kTsluW;
  const int cs2 = cluster_size_for(ctx, ncand);
  const int rp2 = (ncand + cs2 - 1) / cs2;
  if (rp2 > 512 || !cluster_panel_fits_any<float>(kTsluW, rp2))
    return fail(ctx, BEM_ERR_ARG, "too many tournament candidates for one cluster");
  const size_t nprob1 = (size_t)batch * nch;
  int rc = ts_ensure(ctx, L.ts_s, L.ts_cap[0], nprob1 * chunk * kTsluW);
  if (!rc) rc = ts_ensure(ctx, L.ts_ipiv, L.ts_cap[1], nprob1 * chunk);
  if (!rc) rc = ts_ensure(ctx, L.ts_perm, L.ts_cap[2], nprob1 * kPermStride);
  if (!rc) rc = ts_ensure(ctx, L.ts_c, L.ts_cap[3], (size_t)batch * ncand * kTsluW);
  if (!rc) rc = ts_ensure(ctx, L.ts_gid, L.ts_cap[4], (size_t)batch * ncand);
  if (!rc) rc = ts_ensure(ctx, L.ts_cipiv, L.ts_cap[5], (size_t)batch * ncand);
  if (!rc) rc = ts_ensure(ctx, L.ts_cperm, L.ts_cap[6], (size_t)batch * kPermStride);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  // round 1: every chunk of every problem factored on a copy, in one launch
  k_tslu_copy<<<dim3(std::min(64, (chunk * kTsluW + 255) / 256), nch, batch), 256, 0, st>>>(A, lda, bstride, nn, k,
                                                                                         chunk, nch, L.ts_s);
  PanelArgs p1{};
  p1.A = L.ts_s;
  p1.lda = (size_t)chunk;
  p1.bstride = (size_t)chunk * kTsluW;
  p1.nn = chunk;
  p1.k = 0;
  p1.w = kTsluW;
  p1.cs = cs1;
  p1.rp = (chunk + cs1 - 1) / cs1;
  p1.ipiv = L.ts_ipiv;
  p1.ipiv_stride = chunk;
  p1.perm = L.ts_perm;
  p1.perm_stride = kPermStride;
  p1.status = ctx->d_status;
  p1.pstart = nullptr;
  p1.async_mail = ctx->panel_async ? 1 : 0;
  p1.no_singular = 1;
  rc = launch_cluster_panel_any<float>(ctx, p1, (int)nprob1, kTsluW);
  if (rc) return rc;
  // round 2: the chunks' choices, as they are in A, factored the same way
  k_tslu_gather<<<dim3(std::min(64, (ncand * kTsluW + 255) / 256), batch), 256, 0, st>>>(
      A, lda, bstride, nn, k, chunk, nch, L.ts_perm, L.ts_c, L.ts_gid);
  PanelArgs p2 = p1;
  p2.A = L.ts_c;
  p2.lda = (size_t)ncand;
  p2.bstride = (size_t)ncand * kTsluW;
  p2.nn = ncand;
  p2.cs = cs2;
  p2.rp = rp2;
  p2.ipiv = L.ts_cipiv;
  p2.ipiv_stride = ncand;
  p2.perm = L.ts_cperm;
  rc = launch_cluster_panel_any<float>(ctx, p2, batch, kTsluW);
  if (rc) return rc;
  // round 3: the winners to the top in partial pivoting's record, the top
  // block's LU, then L21
  const size_t asmem = (size_t)(2 * kTsluW * kTsluW) * sizeof(zf);
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_tslu_apply), asmem));
  k_tslu_apply<<<batch, 256, asmem, st>>>(A, lda, bstride, nn, k, ncand, L.ts_cperm, L.ts_gid, L.ts_c, L.ipiv, nn,
                                          perm_p, L.pstart, pidx, ctx->d_status);
  const int rows = nn - k - kTsluW;
  if (rows > 0)
    k_tslu_trsm<<<dim3(std::min((rows + 127) / 128, std::max(1, 4 * ctx->num_sms / batch)), batch), 128, 0, st>>>(
        A, lda, bstride, nn, k);
  ctx->launches += 6;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

// One cooperative k_trsv launch over `batch` problems: forward (with the
// interchanges of the last factorisation) and back substitution, or back
// substitution only.
bool make_rows_map(CUtensorMap* m, const void* base, int nn, size_t lda, size_t bstride, int batch, int box_rows);

// The FP32 solves with inverted diagonal blocks (k_tri_inv once per
// factorisation, then k_trsv_f32); done = false when the group's shared
// memory would not fit, and k_trsv runs instead.
constexpr size_t kTrsvF32SmemMax = 200 * 1024;

static int trsv_f32(bem_ctx* ctx, const void* A, size_t lda, size_t bstride, int nn, int batch, void* v,
                    size_t vstride, bool forward, bool& done) {
  LuWork& L = ctx->lu;
  done = false;
  const int npan = (int)L.panels.size(), nblk = (nn + kTrsvBlk - 1) / kTrsvBlk;
  // the largest group (at most 64 CTAs per problem) whose CTAs are all resident
  int group = 0, ldl = 0;
  size_t smem = 0;
  for (int g = std::min(64, std::max(1, nblk)); g >= 1; --g) {
    const int per = (nn + g - 1) / g;
    const int l = (per + 3) & ~1;  // rows of a share rounded out to even ends
    const size_t sm = (size_t)kTrsvBlk * l * sizeof(float2) + (size_t)l * sizeof(int) + 128;
    if (sm > kTrsvF32SmemMax || l > 256) break;  // smaller groups only need more; TMA boxes <= 256 rows
    BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_trsv_f32), sm));
    int occ = 0;
    BEM_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trsv_f32, 256, sm));
    int slots = occ * ctx->num_sms;
    if (ctx->trsv_ctas > 0) slots = std::min(slots, ctx->trsv_ctas);
    if (g * batch <= slots) {
      group = g;
      ldl = l;
      smem = sm;
      break;
    }
  }
  if (!group) return BEM_OK;
  if (!L.tinv_valid) {
    const size_t bytes = (size_t)batch * (npan + nblk) * kTrsvBlk * kTrsvBlk * sizeof(float2);
    if (L.tinv_bytes < bytes) {
      dev_free(ctx, L.tinv);
      L.tinv = nullptr;
      L.tinv_bytes = 0;
      BEM_CUDA(ctx, dev_alloc(ctx, &L.tinv, bytes));
      L.tinv_bytes = bytes;
    }
    ProfScope ps(ctx, 4, 8.0 * (double)(npan + nblk) * kTrsvBlk * kTrsvBlk * kTrsvBlk / 3.0 * batch,
                 2.0 * (double)(npan + nblk) * kTrsvBlk * kTrsvBlk * sizeof(float2) * batch);
    constexpr size_t kInvSmem = (size_t)2 * 64 * 65 * sizeof(float2);
    BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_tri_inv), kInvSmem));
    k_tri_inv<<<dim3(npan + nblk, batch), 64, kInvSmem, ctx->stream>>>(static_cast<const float2*>(A), lda, bstride,
                                                                       nn, npan, L.pstart, L.tinv);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
    L.tinv_valid = true;
  }
  TrsvArgs t{};
  t.A = A;
  t.lda = lda;
  t.bstride = bstride;
  t.nn = nn;
  t.batch = batch;
  t.group = group;
  t.forward = forward ? 1 : 0;
  t.npanels = forward ? npan : 0;
  t.pstart = L.pstart;
  t.perm = L.perm;
  t.v = v;
  t.vstride = vstride;
  t.w = L.trsv_w;
  t.ctr = L.trsv_ctr;
  t.status = ctx->d_status;
  const float2* tinv = L.tinv;
  CUtensorMap tm;
  if (!make_rows_map(&tm, A, nn, lda, bstride, batch, ldl)) return BEM_OK;  // k_trsv instead
  BEM_CUDA(ctx, cudaMemsetAsync(L.trsv_ctr, 0, batch * sizeof(unsigned), ctx->stream));
  void* args[] = {&tm, &t, &tinv, &ldl, const_cast<int*>(&npan)};
  BEM_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)k_trsv_f32, dim3(group * batch), dim3(256), args, smem,
                                            ctx->stream));
  ctx->launches++;
  done = true;
  return BEM_OK;
}

template <typename R>
static int trsv_coop(bem_ctx* ctx, const void* A, size_t lda, size_t bstride, int nn, int batch, void* v,
                     size_t vstride, bool forward) {
  using E = typename Elt<R>::T;
  LuWork& L = ctx->lu;
  const size_t wbytes = (size_t)2 * nn * batch * sizeof(E);
  if (L.trsv_w_bytes < wbytes) {
    dev_free(ctx, L.trsv_w);
    L.trsv_w = nullptr;
    L.trsv_w_bytes = 0;
    BEM_CUDA(ctx, dev_alloc(ctx, &L.trsv_w, wbytes));
    L.trsv_w_bytes = wbytes;
  }
  if (!L.trsv_ctr) BEM_CUDA(ctx, dev_alloc(ctx, &L.trsv_ctr, kMaxBatch * sizeof(unsigned)));
  if (batch < 1 || batch > kMaxBatch) return fail(ctx, BEM_ERR_ARG, "batch size out of range");
  if constexpr (sizeof(R) == 4) {
    if (ctx->trsv_inv) {
      bool done = false;
      const int rc = trsv_f32(ctx, A, lda, bstride, nn, batch, v, vstride, forward, done);
      if (rc || done) return rc;
    }
  }
  const size_t smem = (size_t)kTrsvBlk * kTrsvBlk * sizeof(cpx<R>);
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_trsv<R>), smem));
  int occ = 0;
  BEM_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trsv<R>, 256, smem));
  int slots = occ * ctx->num_sms;
  if (ctx->trsv_ctas > 0) slots = std::min(slots, ctx->trsv_ctas);
  int group = std::min(64, slots / batch);
  group = std::min(group, std::max(1, (nn + kTrsvBlk - 1) / kTrsvBlk));
  if (group < 1) return fail(ctx, BEM_ERR_ARG, "cooperative solve does not fit the device");
  TrsvArgs t{};
  t.A = A;
  t.lda = lda;
  t.bstride = bstride;
  t.nn = nn;
  t.batch = batch;
  t.group = group;
  t.forward = forward ? 1 : 0;
  t.npanels = forward ? (int)L.panels.size() : 0;
  t.pstart = L.pstart;
  t.perm = L.perm;
  t.v = v;
  t.vstride = vstride;
  t.w = L.trsv_w;
  t.ctr = L.trsv_ctr;
  t.status = ctx->d_status;
  BEM_CUDA(ctx, cudaMemsetAsync(L.trsv_ctr, 0, batch * sizeof(unsigned), ctx->stream));
  void* args[] = {&t};
  BEM_CUDA(ctx, cudaLaunchCooperativeKernel((const void*)k_trsv<R>, dim3(group * batch), dim3(256), args, smem,
                                            ctx->stream));
  ctx->launches++;
  return BEM_OK;
}

template <typename R>
static int lu_run(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch) {
  LuWork& L = ctx->lu;
  const int ncols = nn + 1;
  const size_t es = sizeof(cpx<R>);
  const int cs = cluster_size_for(ctx, nn);
  const size_t lsmem = 64 * 64 * es;
  const size_t bsmem = 64 * 64 * es;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_laswp_trsm<R, false>), lsmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_laswp_trsm<R, true>), 2 * lsmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_backsub<R>), bsmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_gemm_f64), kGemmSmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_gemm_tf32), kGemmTf32Smem));
  if (sizeof(R) == 4 && ctx->use_tcgen05) {
    int rc = tc_ensure(ctx, nn, batch);
    if (rc) return rc;
  }
  L.panels.clear();
  L.tinv_valid = false;  // the solves' block inverses belong to the previous factors
  const bool tc = sizeof(R) == 4 && ctx->use_tcgen05;
  // Panel width for m remaining rows: the widest of 64/32/16 whose rows fit
  // one cluster, at most 512 rows per CTA (one row per thread); 0 when the
  // panel needs the cooperative-grid kernel.
  // FP32 (the mixed form) pivots by tournament per 8-column sub-panel.
  const bool calu = sizeof(R) == 4 && ctx->panel_calu;
  auto panel_nb = [&](int m) {
    const int rp_c = (m + cs - 1) / cs;
    if (rp_c <= 512)
      for (int cand : {64, 32, 16})
        if (calu ? calu_panel_fits_any(cand, rp_c) : cluster_panel_fits_any<R>(cand, rp_c)) return cand;
    return 0;
  };
  // Factors the panel starting at column k; returns its width and gather lists.
  auto run_panel = [&](int k, int& w, int*& perm_p) -> int {
    const int m = nn - k;
    perm_p = L.perm + L.panels.size() * (size_t)batch * kPermStride;  // this panel's lists
    PanelArgs pa{};
    pa.A = A;
    pa.lda = lda;
    pa.bstride = bstride;
    pa.nn = nn;
    pa.k = k;
    pa.ipiv = L.ipiv;
    pa.ipiv_stride = nn;
    pa.perm = perm_p;
    pa.perm_stride = kPermStride;
    pa.status = ctx->d_status;
    pa.pstart = L.pstart;
    pa.pidx = (int)L.panels.size();
    pa.async_mail = ctx->panel_async ? 1 : 0;
    const int nb = panel_nb(m);
    ProfScope ps(ctx, 1, 0.0, 2.0 * (double)m * std::min(nb ? nb : 64, m) * es * batch);
    if (nb) {
      w = std::min(nb, m);
      pa.w = w;
      pa.rp = (m + cs - 1) / cs;
      pa.cs = cs;  // CTAs past the last row own no rows but join every barrier
      int rc = calu ? launch_calu_panel_any(ctx, pa, batch, nb) : launch_cluster_panel_any<R>(ctx, pa, batch, nb);
      if (rc) return rc;
      ctx->launches++;
    } else if (sizeof(R) == 4 && ctx->panel_tslu && m > kTsluW) {
      // FP32 panel taller than one cluster holds: tournament pivoting.
      w = kTsluW;
      int rc = tslu_panel(ctx, static_cast<float2*>(A), lda, bstride, nn, k, batch, perm_p, (int)L.panels.size());
      if (rc) return rc;
    } else {
      // Panel taller than one cluster holds: cooperative grid, one problem at a time.
      int G = std::min({ctx->num_sms, kMaxGrid, (m + 15) / 16});
      const int rp = (m + G - 1) / G;
      int nbg = 64;
      if ((size_t)rp * 64 * es > kPanelSmemBudget) nbg = 32;
      if ((size_t)rp * nbg * es > kPanelSmemBudget) return fail(ctx, BEM_ERR_ARG, "matrix too large for the panel kernels");
      w = std::min(nbg, m);
      G = (m + rp - 1) / rp;
      pa.w = w;
      pa.rp = rp;
      pa.cs = G;
      pa.slot_val = L.slot_val;
      pa.slot_row = L.slot_row;
      pa.cand = L.cand;
      pa.drow = L.drow;
      pa.bar = L.barrier;
      for (int b = 0; b < batch; ++b) {
        PanelArgs pb = pa;
        pb.A = static_cast<char*>(A) + (size_t)b * bstride * es;
        pb.ipiv = L.ipiv + (size_t)b * nn;
        pb.perm = perm_p + (size_t)b * kPermStride;
        int rc = (nbg == 64) ? launch_grid_panel<R, 64>(ctx, pb) : launch_grid_panel<R, 32>(ctx, pb);
        if (rc) return rc;
        ctx->launches++;
      }
    }
    BEM_CUDA(ctx, cudaGetLastError());
    L.panels.push_back({k, w});
    return BEM_OK;
  };
  // L11^-1 of the panel at k (for k_laswp_tc) and, for panel gi of a group
  // of gsize, the group's row maps (k_l11_inv).
  auto linv_maps = [&](int k, int w, const int* perm_p, int gi, int gsize) -> int {
    LuWork& LW = ctx->lu;
    const size_t lbytes = (size_t)batch * 64 * 64 * sizeof(float2);
    if (LW.linv_bytes < lbytes) {
      dev_free(ctx, LW.linv);
      LW.linv = nullptr;
      LW.linv_bytes = 0;
      BEM_CUDA(ctx, dev_alloc(ctx, &LW.linv, lbytes));
      LW.linv_bytes = lbytes;
    }
    const size_t mbytes = (size_t)batch * kGroupMaps * nn * sizeof(int);
    if (LW.gmap_bytes < mbytes) {
      dev_free(ctx, LW.gmap);
      LW.gmap = nullptr;
      LW.gmap_bytes = 0;
      BEM_CUDA(ctx, dev_alloc(ctx, &LW.gmap, mbytes));
      LW.gmap_bytes = mbytes;
    }
    BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_l11_inv), (2 * kLtTile)));
    k_l11_inv<<<batch, 1024, 2 * kLtTile, ctx->stream>>>(static_cast<const float2*>(A), lda, bstride, k, w, LW.linv,
                                                         perm_p, kPermStride, LW.gmap, nn, gi, gsize);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
    return BEM_OK;
  };
  // Interchanges + U12 of the panel at k for columns [c0, ncols), packed for
  // the tensor cores at K slot koff (rows c - ubase).  Columns from cdefer
  // on first take the deferred update of the nprev earlier panels of the
  // group (at kfirst, kfirst + 64, ...); gi/gsize: the panel's place in its
  // group (-1: none).
  // pack_r0 >= 0: also pack this panel's L21 (rows pack_r0..) at K slot koff
  // for the update that follows (packed = true when done here).
  auto laswp = [&](int k, int w, int c0, const int* perm_p, int ubase, int koff, int kfirst, int nprev, int cdefer,
                   int gi, int gsize, int pack_r0, bool& packed) -> int {
    packed = false;
    const int cols = ncols - c0;
    if (cols <= 0) return BEM_OK;
    const bool pre = nprev > 0;
    // rows k..k+w-1 (and the displaced rows) of every column read and written once
    ProfScope ps(ctx, 2, 0.0, 2.0 * (double)cols * (2 * w) * es * batch);
    float* ure = tc ? ctx->tc.ure : nullptr;
    float* uim = tc ? ctx->tc.uim : nullptr;
    if (sizeof(R) == 4 && ctx->laswp_tc) {
      int rc = linv_maps(k, w, perm_p, gi, gsize);
      if (rc) return rc;
      // one CTA per SM (registers; shared memory for three or six 64 x 64 tiles)
      const int ntiles = (cols + 63) / 64;
      const int per = std::max(1, ctx->num_sms / batch);
      const int tb = std::min(ntiles, per);
      const size_t sm = (pre ? 6 : 3) * kLtTile;
      float2* A2 = static_cast<float2*>(A);
      LuWork& LW = ctx->lu;
      const int pk = (ure && pack_r0 >= 0) ? pack_r0 : -1;
      float* lhat = ctx->tc.lhat;
      if (pre) {
        BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_laswp_tc<true>), sm));
        k_laswp_tc<true><<<dim3(tb, batch), 256, sm, ctx->stream>>>(
            A2, lda, bstride, k, w, c0, ncols, perm_p, kPermStride, ure, uim, nn + 1, ubase, koff, kfirst, nprev,
            cdefer, LW.gmap, nn, LW.linv, lhat, 2 * nn, pk);
      } else {
        BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_laswp_tc<false>), sm));
        k_laswp_tc<false><<<dim3(tb, batch), 256, sm, ctx->stream>>>(
            A2, lda, bstride, k, w, c0, ncols, perm_p, kPermStride, ure, uim, nn + 1, ubase, koff, kfirst, 0, ncols,
            LW.gmap, nn, LW.linv, lhat, 2 * nn, pk);
      }
      ctx->launches++;
      BEM_CUDA(ctx, cudaGetLastError());
      packed = pk >= 0;
      return BEM_OK;
    }
    if (gi >= 0 && sizeof(R) == 4) {  // the grouped packs read L through the row maps
      int rc = linv_maps(k, w, perm_p, gi, gsize);
      if (rc) return rc;
    }
    // substitution kernel: at most one earlier panel (pairs), deferred everywhere
    const int blocks = std::max(1, std::min((cols + 31) / 32, (4 * ctx->num_sms + batch - 1) / batch));
    if (pre)
      k_laswp_trsm<R, true><<<dim3(blocks, batch), 256, 2 * lsmem, ctx->stream>>>(
          A, lda, bstride, k, w, c0, ncols, perm_p, kPermStride, ure, uim, nn + 1, ubase, koff, kfirst, k - kfirst);
    else
      k_laswp_trsm<R, false><<<dim3(blocks, batch), 256, lsmem, ctx->stream>>>(
          A, lda, bstride, k, w, c0, ncols, perm_p, kPermStride, ure, uim, nn + 1, ubase, koff, kfirst, 0);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
    return BEM_OK;
  };
  for (int k = 0; k < nn;) {
    const int m = nn - k;
    // G = 2 or 4 64-column panels per trailing update (K = 64 G) on the
    // tensor-core path.  Within the group the LU is right-looking: panel i's
    // update of the group's remaining columns is applied at once (a narrow
    // update).  For the columns past the group it is deferred: their rows
    // receive the later panels' interchanges without it, each panel's U rows
    // there first get the earlier panels' deferred update (their L read at
    // this panel's rows through the group's row maps), and the rest is one
    // K = 64 G update whose Lhat takes every earlier panel's L rows through
    // its row map.  A keeps the factors of the one-panel-at-a-time LU (L in
    // panel order), so the solves are unchanged.
    const bool tcg = tc && sizeof(R) == 4;
    // panel width at m remaining rows: the cluster kernels', or 64 for a tall
    // FP32 panel (the tournament and the grid kernel both factor 64 columns
    // of FP32 panels up to 60000 rows), so that tall panels form groups too
    auto pw = [&](int mm) {
      const int nb = panel_nb(mm);
      return nb ? nb : ((sizeof(R) == 4 && mm > kTsluW && mm <= 60000) ? kTsluW : 0);
    };
    const bool fit4 = m > 256 && pw(m) == 64 && pw(m - 64) == 64 && pw(m - 128) == 64 && pw(m - 192) == 64;
    const bool fit2 = m > 128 && pw(m) == 64 && pw(m - 64) == 64;
    const int G = (tcg && ctx->lu_quads && ctx->laswp_tc && fit4) ? 4 : ((tcg && ctx->lu_pairs && fit2) ? 2 : 1);
    if (G > 1) {
      const int kG = k + 64 * G, ubase = k + 64;
      float2* A2 = static_cast<float2*>(A);
      for (int i = 0; i < G; ++i) {
        const int ki = k + 64 * i;
        int wi = 0, *pi = nullptr;
        int rc = run_panel(ki, wi, pi);
        if (rc) return rc;
        bool packed = false;
        rc = laswp(ki, 64, ki + 64, pi, ubase, 64 * i, k, i, kG, i, G, i < G - 1 ? ki + 64 : -1, packed);
        if (rc) return rc;
        if (i < G - 1) {  // panel i's update of the group's remaining columns
          const int r0 = ki + 64;
          ProfScope ps(ctx, 3, 8.0 * (double)(nn - r0) * (double)(kG - r0) * 64.0 * batch,
                       2.0 * (double)(nn - r0) * (double)(kG - r0) * es * batch);
          if (!packed) rc = tc_pack_l(ctx, A2, lda, bstride, nn, ki, 64, r0, 64 * i, batch, nullptr, 0);
          if (!rc) rc = tc_gemm(ctx, A2, lda, bstride, nn, r0, r0, kG, 64, r0 - ubase, batch, 64 * i);
          if (rc) return rc;
        }
      }
      if (kG < nn) {
        ProfScope ps(ctx, 3, 8.0 * (double)(nn - kG) * (double)(ncols - kG) * 64.0 * G * batch,
                     2.0 * (double)(nn - kG) * (double)(ncols - kG) * es * batch);
        // every panel's L at its K slot in one launch, panels 0..G-2 through their row maps
        int rc = tc_pack_l(ctx, A2, lda, bstride, nn, k, 64, kG, 0, batch, ctx->lu.gmap, (size_t)kGroupMaps * nn,
                           G, G - 1);
        if (!rc) rc = tc_gemm(ctx, A2, lda, bstride, nn, kG, kG, ncols, 64 * G, kG - ubase, batch, 0);
        if (rc) return rc;
      }
      k = kG;
      continue;
    }
    // FP64: two panels of the same width nb per trailing update (K = 2 nb).
    // Panel 1's update reaches panel 2's columns at once (a narrow update);
    // past the pair, panel 2's interchanges reach rows that have not taken
    // panel 1's update, panel 2's U rows first take it (k_laswp_trsm<PRE>,
    // panel 1's L read at panel 2's rows through its gather list), and the
    // rest is one K = 2 nb update whose first nb columns read panel 1's L
    // through the same list.  A keeps the factors of the one-panel-at-a-time
    // LU, so the solves are unchanged.
    const int nbp = sizeof(R) == 8 && ctx->f64_pairs ? panel_nb(m) : 0;
    if (nbp > 0 && m > 2 * nbp && panel_nb(m - nbp) == nbp) {
      double2* A2 = static_cast<double2*>(A);
      int w1 = 0, w2 = 0, *p1 = nullptr, *p2 = nullptr;
      int rc = run_panel(k, w1, p1);
      if (rc) return rc;
      const int k2 = k + w1;
      bool packed = false;
      rc = laswp(k, w1, k2, p1, k2, 0, k, 0, k2, -1, 1, -1, packed);
      if (rc) return rc;
      {  // panel 1's update of panel 2's columns
        ProfScope ps(ctx, 3, 8.0 * (double)(nn - k2) * (double)nbp * (double)w1 * batch,
                     2.0 * (double)(nn - k2) * (double)nbp * es * batch);
        if (ctx->f64_cublas) {
          rc = f64_gemm_cublas(ctx, A2, lda, bstride, nn, k, w1, k2, k2, k2 + nbp, batch, nullptr, 0);
          if (rc) return rc;
        } else {
          dim3 grid((nn - k2 + GBM - 1) / GBM, (nbp + GBN - 1) / GBN, batch);
          k_gemm_f64<<<grid, 256, kGemmSmem, ctx->stream>>>(A2, lda, bstride, nn, k, w1, k2, k2, k2 + nbp, nullptr,
                                                           0, 0);
          ctx->launches++;
          BEM_CUDA(ctx, cudaGetLastError());
        }
      }
      rc = run_panel(k2, w2, p2);
      if (rc) return rc;
      const int kG = k2 + w2;
      rc = laswp(k2, w2, kG, p2, kG, 0, k, 1, kG, -1, 1, -1, packed);
      if (rc) return rc;
      if (kG < nn) {
        const int cols = ncols - kG;
        ProfScope ps(ctx, 3, 8.0 * (double)(nn - kG) * (double)cols * (double)(w1 + w2) * batch,
                     2.0 * (double)(nn - kG) * (double)cols * es * batch);
        if (ctx->f64_cublas) {
          // both panels' L in one buffer (the first through the second's
          // gather list), then one ZGEMM with K = w1 + w2
          LuWork& LW = ctx->lu;
          const size_t per = (size_t)(nn - kG) * (w1 + w2), need = per * batch;
          if (LW.lg_cap < need) {
            dev_free(ctx, LW.lg);
            LW.lg = nullptr;
            LW.lg_cap = 0;
            BEM_CUDA(ctx, dev_alloc(ctx, &LW.lg, need * sizeof(double2)));
            LW.lg_cap = need;
          }
          k_gather_l_pair<<<dim3((nn - kG + 255) / 256, batch), 256, 0, ctx->stream>>>(
              A2, lda, bstride, nn, k, w1, w2, kG, p2, kPermStride, LW.lg, per);
          ctx->launches++;
          BEM_CUDA(ctx, cudaGetLastError());
          rc = f64_gemm_cublas(ctx, A2, lda, bstride, nn, k, w1 + w2, kG, kG, ncols, batch, LW.lg, per);
          if (rc) return rc;
        } else {
          dim3 grid((nn - kG + GBM - 1) / GBM, (cols + GBN - 1) / GBN, batch);
          k_gemm_f64<<<grid, 256, kGemmSmem, ctx->stream>>>(A2, lda, bstride, nn, k, w1 + w2, kG, kG, ncols, p2,
                                                           kPermStride, w1);
          ctx->launches++;
          BEM_CUDA(ctx, cudaGetLastError());
        }
      }
      k = kG;
      continue;
    }
    int w = 0, *perm_p = nullptr;
    int rc = run_panel(k, w, perm_p);
    if (rc) return rc;
    const int c0 = k + w;
    if (c0 < ncols) {
      const int cols = ncols - c0;
      bool packed = false;
      rc = laswp(k, w, c0, perm_p, c0, 0, k, 0, c0, -1, 1, tc ? c0 : -1, packed);
      if (rc) return rc;
      if (c0 < nn) {
        ProfScope ps(ctx, 3, 8.0 * (double)(nn - c0) * (double)cols * (double)w * batch,
                     2.0 * (double)(nn - c0) * (double)cols * es * batch);
        if (tc) {
          if (packed)
            rc = tc_gemm(ctx, static_cast<float2*>(A), lda, bstride, nn, c0, c0, nn + 1, w, 0, batch, 0);
          else
            rc = tc_trailing_update(ctx, static_cast<float2*>(A), lda, bstride, nn, k, w, batch);
          if (rc) return rc;
        } else if (sizeof(R) == 8 && ctx->f64_cublas) {
          rc = f64_update_cublas(ctx, static_cast<double2*>(A), lda, bstride, nn, k, w, c0, ncols, batch);
          if (rc) return rc;
        } else if (sizeof(R) == 8) {
          dim3 grid((nn - c0 + GBM - 1) / GBM, (cols + GBN - 1) / GBN, batch);
          k_gemm_f64<<<grid, 256, kGemmSmem, ctx->stream>>>(static_cast<double2*>(A), lda, bstride, nn, k, w, c0, c0,
                                                           ncols, nullptr, 0, 0);
          ctx->launches++;
        } else {
          dim3 grid((nn - c0 + TBM - 1) / TBM, (cols + TBN - 1) / TBN, batch);
          k_gemm_tf32<<<grid, 256, kGemmTf32Smem, ctx->stream>>>(static_cast<float2*>(A), lda, bstride, nn, k, w, c0,
                                                                c0, ncols);
          ctx->launches++;
        }
        BEM_CUDA(ctx, cudaGetLastError());
      }
    }
    k += w;
  }
  ProfScope ps(ctx, 4, 4.0 * (double)nn * nn * batch, 0.5 * (double)nn * nn * es * batch);
  if (ctx->use_trsv_coop) {
    using E = typename Elt<R>::T;
    return trsv_coop<R>(ctx, A, lda, bstride, nn, batch, static_cast<E*>(A) + (size_t)nn * lda, bstride, false);
  }
  const int nblocks = (nn + 63) / 64;
  for (int sblk = nblocks - 1; sblk >= 0; --sblk) {
    const int b0 = sblk * 64;
    k_backsub<R><<<dim3(1 + (b0 + 255) / 256, batch), 256, bsmem, ctx->stream>>>(A, lda, bstride, nn, sblk,
                                                                                  nullptr, 0);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
  }
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// Solves with the stored factors for a new right-hand side v (per problem):
// panel by panel, replay the panel's interchanges on v (one gather), solve
// with the unit lower L11, update the rows below with L21; then the upper
// back substitution.  Used by iterative refinement.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256) k_fwd_panel(void* Av, size_t lda, size_t bstride, void* vv, size_t vstride,
                                                   int k, int w, const int* __restrict__ perm, int perm_stride) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  constexpr int NB = 64;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s_L = reinterpret_cast<C*>(smem_raw);  // [NB][NB]
  __shared__ C s_tmp[2 * NB];
  const int prob = blockIdx.x;
  E* A = static_cast<E*>(Av) + (size_t)prob * bstride;
  E* v = static_cast<E*>(vv) + (size_t)prob * vstride;
  const int* pl = perm + (size_t)prob * perm_stride;
  const int count = pl[0];
  for (int idx = threadIdx.x; idx < w * w; idx += blockDim.x) {
    const int c = idx / w, r = idx % w;
    s_L[c * NB + r] = ldc<R>(&A[(size_t)(k + c) * lda + k + r]);
  }
  for (int e = threadIdx.x; e < count; e += blockDim.x) s_tmp[e] = ldc<R>(&v[pl[2 + 2 * e]]);
  __syncthreads();
  for (int e = threadIdx.x; e < count; e += blockDim.x)
    if (e >= w) stc<R>(&v[pl[1 + 2 * e]], s_tmp[e]);
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  C v0 = lane < w ? s_tmp[lane] : C{R(0), R(0)};
  C v1 = lane + 32 < w ? s_tmp[lane + 32] : C{R(0), R(0)};
  for (int i = 0; i < w; ++i) {
    const C src = (i < 32) ? v0 : v1;
    C ui;
    ui.re = __shfl_sync(0xffffffffu, src.re, i & 31);
    ui.im = __shfl_sync(0xffffffffu, src.im, i & 31);
    if (lane > i && lane < w) cfms(v0, s_L[i * NB + lane], ui);
    if (lane + 32 > i && lane + 32 < w) cfms(v1, s_L[i * NB + lane + 32], ui);
  }
  if (lane < w) stc<R>(&v[k + lane], v0);
  if (lane + 32 < w) stc<R>(&v[k + lane + 32], v1);
}

template <typename R>
__global__ void __launch_bounds__(256) k_fwd_update(void* Av, size_t lda, size_t bstride, void* vv, size_t vstride,
                                                    int k, int w, int nn) {
  using E = typename Elt<R>::T;
  using C = cpx<R>;
  __shared__ C s_x[64];
  E* A = static_cast<E*>(Av) + (size_t)blockIdx.y * bstride;
  E* v = static_cast<E*>(vv) + (size_t)blockIdx.y * vstride;
  for (int i = threadIdx.x; i < w; i += blockDim.x) s_x[i] = ldc<R>(&v[k + i]);
  __syncthreads();
  const int r = k + w + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  C acc = ldc<R>(&v[r]);
  for (int c = 0; c < w; ++c) cfms(acc, ldc<R>(&A[(size_t)(k + c) * lda + r]), s_x[c]);
  stc<R>(&v[r], acc);
}

template <typename R>
static int lu_solve_vec_t(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch, void* v,
                          size_t vstride) {
  LuWork& L = ctx->lu;
  const size_t es = sizeof(cpx<R>);
  const size_t lsmem = 64 * 64 * es;
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_fwd_panel<R>), lsmem));
  BEM_CUDA(ctx, raise_smem_limit(reinterpret_cast<const void*>(k_backsub<R>), lsmem));
  ProfScope ps(ctx, 4, 8.0 * (double)nn * nn * batch, (double)nn * nn * sizeof(cpx<R>) * batch);
  if (ctx->use_trsv_coop) return trsv_coop<R>(ctx, A, lda, bstride, nn, batch, v, vstride, true);
  for (size_t p = 0; p < L.panels.size(); ++p) {
    const int k = L.panels[p].first, w = L.panels[p].second;
    const int* perm_p = L.perm + p * (size_t)batch * kPermStride;
    k_fwd_panel<R><<<batch, 256, lsmem, ctx->stream>>>(A, lda, bstride, v, vstride, k, w, perm_p, kPermStride);
    ctx->launches++;
    if (k + w < nn) {
      k_fwd_update<R><<<dim3((nn - k - w + 255) / 256, batch), 256, 0, ctx->stream>>>(A, lda, bstride, v, vstride,
                                                                                     k, w, nn);
      ctx->launches++;
    }
  }
  const int nblocks = (nn + 63) / 64;
  for (int sblk = nblocks - 1; sblk >= 0; --sblk) {
    const int b0 = sblk * 64;
    k_backsub<R><<<dim3(1 + (b0 + 255) / 256, batch), 256, lsmem, ctx->stream>>>(A, lda, bstride, nn, sblk, v,
                                                                                  vstride);
    ctx->launches++;
  }
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

int lu_solve_vec(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch, void* v, size_t vstride,
                 bool fp32) {
  return fp32 ? lu_solve_vec_t<float>(ctx, A, lda, bstride, nn, batch, v, vstride)
              : lu_solve_vec_t<double>(ctx, A, lda, bstride, nn, batch, v, vstride);
}

int lu_factor_solve(bem_ctx* ctx) {
  int rc = lu_ensure_workspace(ctx, ctx->sys.nn, 1);
  if (rc) return rc;
  return lu_run<double>(ctx, ctx->sys.A, ctx->sys.lda, 0, ctx->sys.nn, 1);
}

int lu_factor_solve_batch(bem_ctx* ctx, void* A, size_t lda, size_t bstride, int nn, int batch, bool fp32) {
  int rc = lu_ensure_workspace(ctx, nn, batch);
  if (rc) return rc;
  return fp32 ? lu_run<float>(ctx, A, lda, bstride, nn, batch) : lu_run<double>(ctx, A, lda, bstride, nn, batch);
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
  BEM_CUDA(ctx, dev_alloc(ctx, &out, (size_t)blocks * threads * sizeof(double)));
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
  dev_free(ctx, out);
  return BEM_OK;
}

// SIMT FMA throughput: 8 independent chains per thread, every result kept.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters) {
  T a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = T(1e-3) * T(threadIdx.x + q + 1);
  const T b = T(0.999) + T(blockIdx.x & 7) * T(1e-6), c = T(1e-7);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = fma(a[q], b, c);
  }
  T sum = T(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) sum += a[q];
  out[blockIdx.x * blockDim.x + threadIdx.x] = sum;
}

template <typename T>
static int measure_fma_t(bem_ctx* ctx, int iters, double* tflops) {
  const int blocks = ctx->num_sms * 8, threads = 256;
  T* out = nullptr;
  cudaEvent_t e0, e1;
  BEM_CUDA(ctx, dev_alloc(ctx, &out, (size_t)blocks * threads * sizeof(T)));
  BEM_CUDA(ctx, cudaEventCreate(&e0));
  BEM_CUDA(ctx, cudaEventCreate(&e1));
  k_fma_peak<T><<<blocks, threads, 0, ctx->stream>>>(out, iters / 8);  // warm-up
  BEM_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  k_fma_peak<T><<<blocks, threads, 0, ctx->stream>>>(out, iters);
  BEM_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
  ctx->launches += 2;
  BEM_CUDA(ctx, cudaEventSynchronize(e1));
  float ms = 0.f;
  BEM_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
  *tflops = 2.0 * 8.0 * (double)blocks * threads * iters / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(ctx, out);
  return BEM_OK;
}

int measure_fma_peaks(bem_ctx* ctx, double* fp64_tflops, double* fp32_tflops) {
  int rc = measure_fma_t<double>(ctx, 4096, fp64_tflops);
  if (rc) return rc;
  return measure_fma_t<float>(ctx, 16384, fp32_tflops);
}

// ---------------------------------------------------------------------------
// Failure-path self-test: the library's two kinds of bounded device wait, each
// on something that never happens, under the context's wait limit.  which = 0:
// an mbarrier armed for 16 bytes of a bulk copy that is never issued (the wait
// of every TMA load); which = 1: a software grid barrier that expects one CTA
// more than the launch has (the wait of the cooperative kernels).  Both give
// up after the limit, record ST_TIMEOUT and return; nothing is in flight.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32) k_wait_selftest(int which, int* status) {
  __shared__ __align__(8) uint64_t s_bar;
  const unsigned long long wlim = wait_limit(status);
  if (which == 0) {
    if (threadIdx.x == 0) {
      mbar_init(&s_bar, 1);
      mbar_expect_tx(&s_bar, 16u);  // the one arrival, and 16 bytes that never come
    }
    __syncthreads();
    const bool ok = mbar_wait(&s_bar, 0, wlim);
    if (!ok && threadIdx.x == 0) atomicExch(&status[ST_TIMEOUT], 1);
  } else {
    unsigned* ctr = reinterpret_cast<unsigned*>(status + ST_SELFTEST_CTR);
    grid_barrier(ctr, 1u, gridDim.x + 1u, status, wlim);
  }
}

int wait_selftest(bem_ctx* ctx, int which) {
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status + ST_SELFTEST_CTR, 0, sizeof(int), ctx->stream));
  k_wait_selftest<<<1, 32, 0, ctx->stream>>>(which, ctx->d_status);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return check_status(ctx);
}

}  // namespace bem
