// assembly.cu -- H/G assembly kernels for sm_100a (FP64 form).
//
// Work decomposition: one thread per (collocation row I, element column J)
// pair, 32 rows per warp so that every warp writes 3 x 32 consecutive
// complex rows of a column (coalesced column-major stores).  A CTA covers 32
// rows and a chunk of JC element columns; the chunk's Gauss points (position
// and weight*|J|, precomputed once per mesh) are staged in shared memory by
// one bulk copy on the TMA engine.  The per-pair quadrature sums are kept in
// factored form (sums of the radial functions times products of the unit
// vector r/|r| and dr/dn), which is algebraically the reference's
// NPG x NPG sum of SOLFUND matrices (src/Nonsingd.for:45-118).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "bem_internal.h"

namespace bem {

struct GaussRule {
  double gi[kMaxNpg], ome[kMaxNpg];
  int npg;
};

// Shape functions, Jacobian and Gauss point of a 4-node element,
// src/Nonsinge.for:47-106 (same block in Nonsingd.for, Sing_de.for,
// Singge.for).  co[k][c]: corner k, coordinate c.
__device__ __forceinline__ void gauss_point(const double co[4][3], double g1, double g2, double& x,
                                            double& y, double& z, double& det) {
  double sp = 1.0 + g2, sm = 1.0 - g2, rp = 1.0 + g1, rm = 1.0 - g1;
  double p0[4] = {-0.25 * sm, 0.25 * sm, 0.25 * sp, -0.25 * sp};
  double p1[4] = {-0.25 * rm, -0.25 * rp, 0.25 * rp, 0.25 * rm};
  double f[4] = {0.25 * rm * sm, 0.25 * rp * sm, 0.25 * rp * sp, 0.25 * rm * sp};
  double xj0[3], xj1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      t0 = t0 + p0[k] * co[k][c];
      t1 = t1 + p1[k] * co[k][c];
    }
    xj0[c] = t0;
    xj1[c] = t1;
  }
  double d1 = xj0[1] * xj1[2] - xj1[1] * xj0[2];
  double d2 = xj1[0] * xj0[2] - xj0[0] * xj1[2];
  double d3 = xj0[0] * xj1[1] - xj1[0] * xj0[1];
  det = sqrt(d1 * d1 + d2 * d2 + d3 * d3);
  x = y = z = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x = x + co[k][0] * f[k];
    y = y + co[k][1] * f[k];
    z = z + co[k][2] * f[k];
  }
}

// Per element and Gauss point: position and weight ome(ig)*ome(jg)*DET.
// Flags: flags[0] |= 1 if any element (of n) is degenerate, flags[1] for
// the boundary elements (J < nbe) only.
__global__ void k_geometry(int n, int nbe, const double* __restrict__ cx, const double* __restrict__ cy,
                           const double* __restrict__ cz, const int* __restrict__ cone,
                           const double* __restrict__ etas, const double* __restrict__ cxm,
                           const double* __restrict__ cym, const double* __restrict__ czm,
                           GaussRule rule, double4* gq, double4* eta, double4* colloc, double* corner,
                           int* degen, int* flags) {
  const int ng = rule.npg * rule.npg;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * ng) return;
  const int j = (int)(t / ng), g = (int)(t % ng);
  const int jg = g / rule.npg, ig = g % rule.npg;  // JG outer, IG inner
  double co[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int nk = cone[(size_t)k * n + j] - 1;
    co[k][0] = cx[nk];
    co[k][1] = cy[nk];
    co[k][2] = cz[nk];
  }
  double x, y, z, det;
  gauss_point(co, rule.gi[ig], rule.gi[jg], x, y, z, det);
  gq[(size_t)j * ng + g] = make_double4(x, y, z, rule.ome[ig] * rule.ome[jg] * det);
  if (det < 1.0e-5) {
    degen[j] = 1;
    atomicOr(&flags[0], 1);
    if (j < nbe) atomicOr(&flags[1], 1);
  }
  if (g == 0) {
    eta[j] = make_double4(etas[3 * j], etas[3 * j + 1], etas[3 * j + 2], 0.0);
    colloc[j] = make_double4(cxm[j], cym[j], czm[j], 0.0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) corner[(size_t)j * 12 + 3 * k + c] = co[k][c];
  }
}

// ---------------------------------------------------------------------------
// Static Kelvin traction kernel T (src/Solfune.for:18-31) over NBE x N pairs,
// summed per collocation row for the rigid-body diagonal
// (src/Ghmatece.for:258-282).  Thread = row I, loop over the chunk's J.
// Per pair and Gauss point: T_ij = C3/r^2 (drn (C4 d_ij + 3 rd_i rd_j)
//   + C4 (rd_j n_i - rd_i n_j)); sums of the scalar factors are formed per
// element, then combined with the element normal n.
// ---------------------------------------------------------------------------
struct StaticParams {
  int n, nbe, ng, jc;
  double c3, c4;
  const double4* gq;
  const double4* eta;
  const double4* colloc;
  double* part;       // [chunks][nbe][9]
  double* hest_full;  // optional 3nbe x 3n column-major
};

__global__ void __launch_bounds__(128) k_static_rows(StaticParams p) {
  __shared__ double s_sum[4][32][9];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int I = blockIdx.x * 32 + lane;
  const int J0 = blockIdx.y * p.jc;
  const int jn = min(p.jc, p.n - J0);
  double h[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) h[k] = 0.0;
  if (I < p.nbe) {
    const double4 P = p.colloc[I];
    for (int jl = w; jl < jn; jl += 4) {
      const int J = J0 + jl;
      if (J == I) continue;  // HEST(JJ:JJ+2,JJ:JJ+2) = 0 (Ghmatece.for:134-135)
      const double4 nv = p.eta[J];
      const double4* q = p.gq + (size_t)J * p.ng;
      double a0 = 0, b00 = 0, b01 = 0, b02 = 0, b11 = 0, b12 = 0, b22 = 0, c0 = 0, c1 = 0, c2 = 0;
      for (int g = 0; g < p.ng; ++g) {
        const double4 qq = q[g];
        double r1 = qq.x - P.x, r2 = qq.y - P.y, r3 = qq.z - P.z;
        double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
        double ir = 1.0 / r;
        double d0 = r1 * ir, d1 = r2 * ir, d2 = r3 * ir;
        double drn = (r1 * nv.x + r2 * nv.y + r3 * nv.z) * ir;
        double s = qq.w * p.c3 * ir * ir;
        double sd = 3.0 * s * drn;
        a0 = fma(s * p.c4, drn, a0);
        b00 = fma(sd * d0, d0, b00);
        b01 = fma(sd * d0, d1, b01);
        b02 = fma(sd * d0, d2, b02);
        b11 = fma(sd * d1, d1, b11);
        b12 = fma(sd * d1, d2, b12);
        b22 = fma(sd * d2, d2, b22);
        double sc = s * p.c4;
        c0 = fma(sc, d0, c0);
        c1 = fma(sc, d1, c1);
        c2 = fma(sc, d2, c2);
      }
      const double nn_[3] = {nv.x, nv.y, nv.z};
      const double cc[3] = {c0, c1, c2};
      const double bb[3][3] = {{b00, b01, b02}, {b01, b11, b12}, {b02, b12, b22}};
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          double t = (i == j ? a0 : 0.0) + bb[i][j] + nn_[i] * cc[j] - nn_[j] * cc[i];
          h[3 * j + i] += t;
          if (p.hest_full)
            p.hest_full[(size_t)(3 * J + j) * (3 * p.nbe) + 3 * I + i] = t;
        }
    }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) s_sum[w][lane][k] = h[k];
  __syncthreads();
  for (int t = threadIdx.x; t < 32 * 9; t += blockDim.x) {
    const int l = t / 9, k = t % 9;
    const int row = blockIdx.x * 32 + l;
    if (row < p.nbe) {
      double v = ((s_sum[0][l][k] + s_sum[1][l][k]) + s_sum[2][l][k]) + s_sum[3][l][k];
      p.part[((size_t)blockIdx.y * p.nbe + row) * 9 + k] = v;
    }
  }
}

// HESTdiag(:,:,I) = -sum over chunks (fixed order: deterministic).
__global__ void k_static_reduce(int nbe, int chunks, const double* __restrict__ part, double* hestdiag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbe * 9) return;
  double acc = 0.0;
  for (int c = 0; c < chunks; ++c) acc -= part[(size_t)c * nbe * 9 + t];
  hestdiag[t] = acc;
}

// GEST_SINGULAR on the device (src/Ghmatece.for:288-323, src/Singge.for:11-202):
// per element, 4 triangles with corners 3 and 4 collapsed to the centroid,
// each integrated with NPG x NPG points of the Kelvin U kernel
// U_ij = C1/r (C2 d_ij + rd_i rd_j).
__global__ void k_gest(int nbe, const double* __restrict__ corner, const double4* __restrict__ colloc,
                       GaussRule rule, double c1, double c2, double* gestdiag, int* status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nbe) return;
  const double4 P = colloc[j];
  double el[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) el[k][c] = corner[(size_t)j * 12 + 3 * k + c];
  double gsum[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) gsum[k] = 0.0;
  for (int it = 0; it < 4; ++it) {
    double co[4][3];
    const int a = it, b = (it + 1) & 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      co[0][c] = el[a][c];
      co[1][c] = el[b][c];
    }
    co[2][0] = co[3][0] = P.x;
    co[2][1] = co[3][1] = P.y;
    co[2][2] = co[3][2] = P.z;
    double gp[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gp[k] = 0.0;
    for (int jg = 0; jg < rule.npg; ++jg)
      for (int ig = 0; ig < rule.npg; ++ig) {
        double x, y, z, det;
        gauss_point(co, rule.gi[ig], rule.gi[jg], x, y, z, det);
        if (det < 1.0e-5) atomicOr(&status[ST_DEGENERATE], 1);
        double p12 = rule.ome[ig] * rule.ome[jg] * det;
        double r1 = x - P.x, r2 = y - P.y, r3 = z - P.z;
        double r = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
        double rd[3] = {r1 / r, r2 / r, r3 / r};
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
#pragma unroll
          for (int ii = 0; ii < 3; ++ii)
            gp[3 * jj + ii] += ((c1 / r) * (c2 * (ii == jj ? 1.0 : 0.0) + rd[ii] * rd[jj])) * p12;
      }
#pragma unroll
    for (int k = 0; k < 9; ++k) gsum[k] = gsum[k] + gp[k];
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) gestdiag[(size_t)j * 9 + k] = gsum[k];
}

// ---------------------------------------------------------------------------
// Dynamic assembly.
// ---------------------------------------------------------------------------
struct DynCore {
  int nbe, nn, ng, jc, chunks;
  size_t lda;
  size_t a_stride;  // elements between the systems of consecutive problems
  double2 zge;
  double c1, c2, c3, c4;
  int fast_singular;
  const double4* gq;
  const double4* eta;
  const double4* colloc;
  const double* hestdiag;
  const double* gestdiag;
  const int* kode;
  const double2* zdfi;
  double2* A;       // problem b: A + b*a_stride, nn x (nn+1)
  float2* A32;      // optional complex64 copy (same layout)
  double2* zh_pre;  // optional, problem 0 only
  double2* zg_pre;  // optional, problem 0 only
  double2* G;       // optional post-swap G (multiplies ZDFI), same layout as A
  double2* diag_h;  // [batch][nbe][9]
  double2* diag_g;
  double2* rhs_part;  // [batch][chunks][nn]
  int* status;
};
// One mesh, `batch` frequencies (bem_ghmatecd, bem_sweep).
struct DynParams : DynCore {
  StokesConsts<double> kb[kMaxBatch];  // per problem (frequency)
};
// One problem of a grouped launch (bem_batch_solve): its own mesh, BCs and
// constants; its system is padded to npad unknowns, the right-hand side in
// column npad.
struct DynProblem : DynCore {
  StokesConsts<double> kc;
  int npad;
};

__device__ __forceinline__ zd ld(const double2* p) {
  double2 v = *p;
  return zd{v.x, v.y};
}
__device__ __forceinline__ void st(double2* p, zd z) { *p = make_double2(z.re, z.im); }

// Diagonal blocks (I == J): SING_DE (src/Sing_de.for:13-113) with SOLFUNDIF
// (src/Solfundif.for:18-69), Stokes minus Kelvin per Gauss point, plus the
// static diagonals (src/Ghmatecd.for:150-153).  One thread per element.
__device__ __forceinline__ void dyn_diag_body(const DynCore& p, const StokesConsts<double>& kc, int prob) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= p.nbe) return;
  double2* diag_h = p.diag_h + (size_t)prob * p.nbe * 9;
  double2* diag_g = p.diag_g + (size_t)prob * p.nbe * 9;
  const double4 P = p.colloc[j];
  const double4 nv = p.eta[j];
  const double rn0 = nv.x, rn1 = nv.y, rn2 = nv.z;
  zd zh[9], zg[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) zh[k] = zg[k] = zd{0.0, 0.0};
  const double4* q = p.gq + (size_t)j * p.ng;
  for (int g = 0; g < p.ng; ++g) {
    const double4 qq = q[g];
    double r1 = qq.x - P.x, r2 = qq.y - P.y, r3 = qq.z - P.z;
    const double ir = rsqrt(fma(r1, r1, fma(r2, r2, r3 * r3)));  // r and 1/r from one rsqrt
    const double r = fma(r1, r1, fma(r2, r2, r3 * r3)) * ir;
    double drn = (r1 * rn0 + r2 * rn1 + r3 * rn2) * ir;
    const double rd[3] = {r1 * ir, r2 * ir, r3 * ir};
    const double rn[3] = {rn0, rn1, rn2};
    StokesRadial<double> s = stokes_radial(kc, r, ir);
#pragma unroll
    for (int jj = 0; jj < 3; ++jj)
#pragma unroll
      for (int ii = 0; ii < 3; ++ii) {
        const double dl = (ii == jj) ? 1.0 : 0.0;
        zd u = kc.zc0 * (s.fhi * dl - s.cappa * (rd[jj] * rd[ii]));
        zd t = kc.inv4pi * ((s.aa * (drn * dl + rd[jj] * rn[ii])) + s.bb * (rd[ii] * rd[jj] * drn) +
                            s.cc * (rd[ii] * rn[jj]));
        if (p.fast_singular) {
          u.re -= (p.c1 / r) * (p.c2 * dl + rd[ii] * rd[jj]);
          t.re -= (p.c3 * ir * ir) * (drn * (p.c4 * dl + 3.0 * rd[ii] * rd[jj]) +
                                      p.c4 * (rd[jj] * rn[ii] - rd[ii] * rn[jj]));
        }
        cfma(zh[3 * jj + ii], t, qq.w);
        cfma(zg[3 * jj + ii], u, qq.w);
      }
  }
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    if (p.fast_singular) {
      zg[k].re += p.gestdiag[(size_t)j * 9 + k];
      zh[k].re += p.hestdiag[(size_t)j * 9 + k];
    }
    st(&diag_h[(size_t)j * 9 + k], zh[k]);
    st(&diag_g[(size_t)j * 9 + k], zg[k]);
  }
}

__global__ void __launch_bounds__(128) k_dyn_diag(DynParams p) { dyn_diag_body(p, p.kb[blockIdx.z], blockIdx.z); }

// Grouped form: blockIdx.z is the problem; its descriptor is in global memory.
__global__ void __launch_bounds__(128) k_dyn_diag_grp(const DynProblem* __restrict__ g) {
  const DynProblem& p = g[blockIdx.z];
  const StokesConsts<double> kc = p.kc;
  dyn_diag_body(p, kc, 0);
}

// Off-diagonal pairs with the boundary-condition swap (src/Ghmatecd.for:316-333
// as called at :168: column j with KODE=0 gets H <- -G, G <- -H*ZGE) and the
// right-hand side ZFI = G*ZDFI (src/Ghmatecd.for:172-181) fused; G itself is
// not stored.  Diagonal pairs take their blocks from k_dyn_diag.
constexpr int kRowsPerCta = 32;

// Packed index of a symmetric 3x3 entry: 00 01 02 11 12 22.
__host__ __device__ constexpr int sym3(int i, int j) {
  return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5)) : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}
constexpr int kWarpsPerCta = 4;

__device__ __forceinline__ void dyn_offdiag_body(const DynCore& p, const StokesConsts<double>& kc, int prob) {
  extern __shared__ __align__(128) double4 s_gq[];  // [jc][ng]
  __shared__ uint64_t s_bar;
  __shared__ zd s_rhs[kWarpsPerCta][3 * kRowsPerCta];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int I = blockIdx.x * kRowsPerCta + lane;
  const int J0 = blockIdx.y * p.jc;
  // a grouped launch covers its largest member: CTAs past this one's rows or
  // element columns leave at once (uniform per CTA, before any barrier)
  if (J0 >= p.nbe || (int)blockIdx.x * kRowsPerCta >= p.nbe) return;
  const int jn = min(p.jc, p.nbe - J0);
  double2* A = p.A + (size_t)prob * p.a_stride;
  float2* A32 = p.A32 ? p.A32 + (size_t)prob * p.a_stride : nullptr;
  double2* Gp = p.G ? p.G + (size_t)prob * p.a_stride : nullptr;
  const double2* diag_h = p.diag_h + (size_t)prob * p.nbe * 9;
  const double2* diag_g = p.diag_g + (size_t)prob * p.nbe * 9;
  const bool preswap = p.zh_pre && prob == 0;

  if (threadIdx.x == 0) mbar_init(&s_bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned bytes = (unsigned)(jn * p.ng * sizeof(double4));
    mbar_expect_tx(&s_bar, bytes);
    bulk_g2s(s_gq, p.gq + (size_t)J0 * p.ng, bytes, &s_bar);
  }
  const unsigned long long wlim = wait_limit(p.status);
  if (!mbar_wait(&s_bar, 0, wlim)) {
    if (threadIdx.x == 0) atomicExch(&p.status[ST_TIMEOUT], 1);
    mbar_wait(&s_bar, 0, wlim);  // let the copy in flight land before leaving
    return;
  }

  const bool valid = I < p.nbe;
  const double4 P = valid ? p.colloc[I] : make_double4(0.0, 0.0, 0.0, 0.0);
  zd rhs[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};

  for (int jl = w; jl < jn; jl += kWarpsPerCta) {
    const int J = J0 + jl;
    const double4 nv = p.eta[J];
    const double n3[3] = {nv.x, nv.y, nv.z};
    zd U[3][3], T[3][3];  // [i][j]: row component i, column component j
    if (valid && J != I) {
      zd F{0, 0}, A0{0, 0};
      zd K[6], B[6], A1[3], C[3];
#pragma unroll
      for (int k = 0; k < 6; ++k) K[k] = B[k] = zd{0, 0};
#pragma unroll
      for (int k = 0; k < 3; ++k) A1[k] = C[k] = zd{0, 0};
      const double4* q = s_gq + jl * p.ng;
#pragma unroll 2
      for (int g = 0; g < p.ng; ++g) {
        const double4 qq = q[g];
        const double r1 = qq.x - P.x, r2 = qq.y - P.y, r3 = qq.z - P.z;
        const double rr = fma(r1, r1, fma(r2, r2, r3 * r3));
        const double ir = rsqrt(rr);  // r and 1/r from one rsqrt
        const double r = rr * ir;
        const double d0 = r1 * ir, d1 = r2 * ir, d2 = r3 * ir;
        const double drn = (r1 * n3[0] + r2 * n3[1] + r3 * n3[2]) * ir;
        const StokesRadial<double> s = stokes_radial(kc, r, ir);
        const double wt = qq.w;
        const double w0 = wt * d0, w1 = wt * d1, w2 = wt * d2, wd = wt * drn;
        cfma(F, s.fhi, wt);
        cfma(K[0], s.cappa, w0 * d0);
        cfma(K[1], s.cappa, w0 * d1);
        cfma(K[2], s.cappa, w0 * d2);
        cfma(K[3], s.cappa, w1 * d1);
        cfma(K[4], s.cappa, w1 * d2);
        cfma(K[5], s.cappa, w2 * d2);
        cfma(A0, s.aa, wd);
        cfma(A1[0], s.aa, w0);
        cfma(A1[1], s.aa, w1);
        cfma(A1[2], s.aa, w2);
        const double e0 = wd * d0, e1 = wd * d1, e2 = wd * d2;
        cfma(B[0], s.bb, e0 * d0);
        cfma(B[1], s.bb, e0 * d1);
        cfma(B[2], s.bb, e0 * d2);
        cfma(B[3], s.bb, e1 * d1);
        cfma(B[4], s.bb, e1 * d2);
        cfma(B[5], s.bb, e2 * d2);
        cfma(C[0], s.cc, w0);
        cfma(C[1], s.cc, w1);
        cfma(C[2], s.cc, w2);
      }
      // U_ij = c0 (d_ij F - K_ij); T_ij = (d_ij A0 + n_i A1_j + B_ij + n_j C_i) / 4pi.
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const int sy = sym3(i, j);
          zd u = (i == j) ? F - K[sy] : -K[sy];
          U[i][j] = kc.zc0 * u;
          zd t = B[sy];
          cfma(t, A1[j], n3[i]);
          cfma(t, C[i], n3[j]);
          if (i == j) t = t + A0;
          T[i][j] = t * kc.inv4pi;
        }
    } else if (valid) {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          U[i][j] = ld(&diag_g[(size_t)J * 9 + 3 * j + i]);
          T[i][j] = ld(&diag_h[(size_t)J * 9 + 3 * j + i]);
        }
    }
    if (valid) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int col = 3 * J + j;
        const int kd = p.kode[col];
        const zd x = ld(&p.zdfi[col]);
        const zd ge{p.zge.x, p.zge.y};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const size_t row = (size_t)3 * I + i;
          zd h = T[i][j], g = U[i][j];
          if (preswap) {
            st(&p.zh_pre[(size_t)col * p.nn + row], h);
            st(&p.zg_pre[(size_t)col * p.nn + row], g);
          }
          if (kd == 0) {
            zd hg = h * ge;
            h = -g;
            g = -hg;
          }
          st(&A[(size_t)col * p.lda + row], h);
          if (A32) A32[(size_t)col * p.lda + row] = make_float2((float)h.re, (float)h.im);
          if (Gp) st(&Gp[(size_t)col * p.lda + row], g);
          cfma(rhs[i], g, x);
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) s_rhs[w][3 * lane + i] = rhs[i];
  __syncthreads();
  for (int t = threadIdx.x; t < 3 * kRowsPerCta; t += blockDim.x) {
    const int row = 3 * blockIdx.x * kRowsPerCta + t;
    if (row < p.nn) {
      zd acc = s_rhs[0][t];
#pragma unroll
      for (int v = 1; v < kWarpsPerCta; ++v) acc = acc + s_rhs[v][t];
      st(&p.rhs_part[((size_t)prob * p.chunks + blockIdx.y) * p.nn + row], acc);
    }
  }
}

__global__ void __launch_bounds__(128) k_dyn_offdiag(DynParams p) {
  dyn_offdiag_body(p, p.kb[blockIdx.z], blockIdx.z);
}

__global__ void __launch_bounds__(128) k_dyn_offdiag_grp(const DynProblem* __restrict__ g) {
  const DynProblem& p = g[blockIdx.z];
  dyn_offdiag_body(p, p.kc, 0);
}

// Grouped form of the right-hand-side reduction and the padding of a class
// (blockIdx.y = problem): the RHS (chunk partials summed in chunk order, as
// k_rhs_reduce) goes to column npad with zeros below row nn; columns < nn
// get zero rows nn..npad-1; columns nn..npad-1 become the identity.  The
// padding never pivots and stays untouched by the updates.
__global__ void __launch_bounds__(256) k_rhs_pad_grp(const DynProblem* __restrict__ g) {
  const DynProblem& p = g[blockIdx.y];
  const int n = p.nn, npad = p.npad, e = npad - n, chunks = p.chunks;
  const size_t lda = p.lda;
  double2* A = p.A;
  float2* A32 = p.A32;
  const double2* part = p.rhs_part;
  const long long live = (long long)e * n, total = (long long)npad + live + (long long)e * npad;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int row, col;
    zd v{0.0, 0.0};
    if (i < npad) {
      row = (int)i;
      col = npad;
      if (row < n)
        for (int c = 0; c < chunks; ++c) v = v + ld(&part[(size_t)c * n + row]);
    } else if (i < npad + live) {
      const long long k = i - npad;
      col = (int)(k / e);
      row = n + (int)(k % e);
    } else {
      const long long k = i - npad - live;
      col = n + (int)(k / npad);
      row = (int)(k % npad);
      if (row == col) v.re = 1.0;
    }
    const size_t idx = (size_t)col * lda + row;
    st(&A[idx], v);
    if (A32) A32[idx] = make_float2((float)v.re, (float)v.im);
  }
}

// RHS column of A: sum of the per-chunk partials in chunk order.
__global__ void k_rhs_reduce(int nn, int chunks, size_t lda, size_t a_stride, const double2* __restrict__ part,
                             double2* A, float2* A32) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  const int prob = blockIdx.y;
  const double2* pp = part + (size_t)prob * chunks * nn;
  zd acc{0.0, 0.0};
  for (int c = 0; c < chunks; ++c) acc = acc + ld(&pp[(size_t)c * nn + r]);
  const size_t idx = (size_t)prob * a_stride + (size_t)nn * lda + r;
  st(&A[idx], acc);
  if (A32) A32[idx] = make_float2((float)acc.re, (float)acc.im);
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
static int jc_for(int ng) { return std::max(1, std::min(64, 1024 / ng)); }

int launch_geometry(bem_ctx* ctx, const double* d_cx, const double* d_cy, const double* d_cz,
                    const int* d_cone, const double* d_etas, const double* d_cxm, const double* d_cym,
                    const double* d_czm) {
  Mesh& m = ctx->mesh;
  GaussRule rule{};
  rule.npg = m.npg;
  for (int i = 0; i < m.npg; ++i) {
    rule.gi[i] = m.gi[i];
    rule.ome[i] = m.ome[i];
  }
  int* d_flags = ctx->d_status + ST_COUNT;  // two mesh flags after the status words
  BEM_CUDA(ctx, cudaMemsetAsync(d_flags, 0, 2 * sizeof(int), ctx->stream));
  BEM_CUDA(ctx, cudaMemsetAsync(m.degen, 0, m.n * sizeof(int), ctx->stream));
  const long long total = (long long)m.n * m.ng;
  const int threads = 256;
  k_geometry<<<(unsigned)((total + threads - 1) / threads), threads, 0, ctx->stream>>>(
      m.n, m.nbe, d_cx, d_cy, d_cz, d_cone, d_etas, d_cxm, d_cym, d_czm, rule, m.gq, m.eta, m.colloc,
      m.corner, m.degen, d_flags);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

int launch_static(bem_ctx* ctx, const double c[4], int compute_gest, double* hest_full) {
  Mesh& m = ctx->mesh;
  const int jc = jc_for(m.ng);
  const int chunks = (m.n + jc - 1) / jc;
  // static_chunks holds the capacity of static_part in chunks of nbe*9 doubles
  // for the current mesh (reset to 0 by bem_mesh_upload).
  if (chunks > ctx->static_chunks) {
    if (ctx->static_part) dev_free(ctx, ctx->static_part);
    ctx->static_part = nullptr;
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->static_part, (size_t)chunks * m.nbe * 9 * sizeof(double)));
    ctx->static_chunks = chunks;
  }
  StaticParams p{};
  p.n = m.n;
  p.nbe = m.nbe;
  p.ng = m.ng;
  p.jc = jc;
  p.c3 = c[2];
  p.c4 = c[3];
  p.gq = m.gq;
  p.eta = m.eta;
  p.colloc = m.colloc;
  p.part = ctx->static_part;
  p.hest_full = hest_full;
  dim3 grid((m.nbe + kRowsPerCta - 1) / kRowsPerCta, chunks);
  k_static_rows<<<grid, 128, 0, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  k_static_reduce<<<(m.nbe * 9 + 255) / 256, 256, 0, ctx->stream>>>(m.nbe, chunks, ctx->static_part,
                                                                     ctx->hestdiag);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  if (compute_gest) {
    GaussRule rule{};
    rule.npg = m.npg;
    for (int i = 0; i < m.npg; ++i) {
      rule.gi[i] = m.gi[i];
      rule.ome[i] = m.ome[i];
    }
    k_gest<<<(m.nbe + 127) / 128, 128, 0, ctx->stream>>>(m.nbe, m.corner, m.colloc, rule, c[0], c[1],
                                                         ctx->gestdiag, ctx->d_status);
    ctx->launches++;
    BEM_CUDA(ctx, cudaGetLastError());
  }
  return BEM_OK;
}

StokesConsts<double> make_consts(const double zge_[2], const double zcs_[2],
                                        const double zcp_[2], double fr) {
  // Solfund.for:29-35 in double on the host.
  auto mul = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
  auto div = [](double2 a, double2 b) {
    double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
  };
  const double pi = 4.0 * std::atan(1.0);
  double2 zge = make_double2(zge_[0], zge_[1]);
  double2 zcs = make_double2(zcs_[0], zcs_[1]);
  double2 zcp = make_double2(zcp_[0], zcp_[1]);
  double2 zwi = make_double2(0.0, fr);
  double2 mzwi = make_double2(-zwi.x, -zwi.y);
  StokesConsts<double> k{};
  double2 c0 = div(make_double2(1.0, 0.0), mul(make_double2(4.0 * pi, 0.0), zge));
  double2 pc = div(zcp, zcs), sc = div(zcs, zcp);
  double2 c1 = mul(pc, pc), c2 = mul(sc, sc);
  double2 kp = div(mzwi, zcp), ks = div(mzwi, zcs);
  k.zkp = zd{kp.x, kp.y};
  k.zks = zd{ks.x, ks.y};
  k.zc2 = zd{c2.x, c2.y};
  k.zc1m2 = zd{c1.x - 2.0, c1.y};
  k.zc0 = zd{c0.x, c0.y};
  k.inv4pi = 1.0 / (4.0 * pi);
  const double2 ikp = div(make_double2(1.0, 0.0), kp), iks = div(make_double2(1.0, 0.0), ks);
  k.izkp = zd{ikp.x, ikp.y};
  k.izks = zd{iks.x, iks.y};
  return k;
}

static DynCore dyn_core(bem_ctx* ctx, const DynBatch& b) {
  Mesh& m = ctx->mesh;
  const int jc = jc_for(m.ng);
  const int chunks = (m.nbe + jc - 1) / jc;
  DynCore p{};
  p.nbe = m.nbe;
  p.nn = 3 * m.nbe;
  p.ng = m.ng;
  p.jc = jc;
  p.chunks = chunks;
  p.lda = b.lda;
  p.a_stride = b.a_stride;
  p.zge = make_double2(b.zge[0], b.zge[1]);
  p.c1 = b.c[0];
  p.c2 = b.c[1];
  p.c3 = b.c[2];
  p.c4 = b.c[3];
  p.fast_singular = (b.flags & BEM_FAST_SINGULAR) ? 1 : 0;
  p.gq = m.gq;
  p.eta = m.eta;
  p.colloc = m.colloc;
  p.hestdiag = ctx->hestdiag;
  p.gestdiag = ctx->gestdiag;
  p.kode = ctx->kode;
  p.zdfi = ctx->zdfi;
  p.A = b.A;
  p.A32 = b.A32;
  p.zh_pre = b.zh_pre;
  p.zg_pre = b.zg_pre;
  p.diag_h = b.diag_h;
  p.diag_g = b.diag_g;
  p.rhs_part = b.rhs_part;
  p.G = b.G;
  p.status = ctx->d_status;
  return p;
}

static DynParams dyn_params(bem_ctx* ctx, const DynBatch& b) {
  DynParams p{};
  static_cast<DynCore&>(p) = dyn_core(ctx, b);
  for (int i = 0; i < b.batch; ++i) p.kb[i] = make_consts(b.zge, b.zcs, b.zcp, b.freqs[i]);
  return p;
}

size_t dyn_problem_bytes() { return sizeof(DynProblem); }

int launch_dynamic_group(bem_ctx* wk, const GroupMember* mem, int count, void* h_desc, void* d_desc) {
  if (count < 1 || count > 65535) return fail(wk, BEM_ERR_ARG, "group size out of range");
  DynProblem* hd = static_cast<DynProblem*>(h_desc);
  int max_nbe = 0, max_chunks = 0;
  long long max_pad = 0;
  size_t smem = 0;
  double work = 0.0, bytes = 0.0;
  for (int i = 0; i < count; ++i) {
    const GroupMember& g = mem[i];
    bem_ctx* pc = g.pc;
    std::lock_guard<std::mutex> lk(pc->mu);
    DynBatch b{};
    b.zge = g.zge;
    b.zcs = g.zcs;
    b.zcp = g.zcp;
    b.c = g.c;
    b.freqs = &g.fr;
    b.batch = 1;
    b.flags = BEM_FAST_SINGULAR;
    b.A = g.A;
    b.lda = g.lda;
    b.a_stride = 0;
    b.A32 = g.A32;
    b.diag_h = g.diag_h;
    b.diag_g = g.diag_g;
    b.rhs_part = g.rhs_part;
    DynProblem q{};
    static_cast<DynCore&>(q) = dyn_core(pc, b);
    q.status = wk->d_status;  // the group reports through the worker
    q.kc = make_consts(g.zge, g.zcs, g.zcp, g.fr);
    q.npad = g.npad;
    if (q.npad < q.nn) return fail(wk, BEM_ERR_ARG, "padded size below the problem size");
    hd[i] = q;
    const Mesh& m = pc->mesh;
    max_nbe = std::max(max_nbe, m.nbe);
    max_chunks = std::max(max_chunks, q.chunks);
    smem = std::max(smem, (size_t)q.jc * m.ng * sizeof(double4));
    const long long e = q.npad - q.nn;
    max_pad = std::max(max_pad, (long long)q.npad + e * q.nn + e * q.npad);
    work += (double)m.nbe * (double)m.nbe * (double)m.ng;
    bytes += (double)q.nn * (q.nn + 1) * (16.0 + (g.A32 ? 8.0 : 0.0));
  }
  const DynProblem* dd = static_cast<const DynProblem*>(d_desc);
  BEM_CUDA(wk, cudaMemcpyAsync(d_desc, hd, (size_t)count * sizeof(DynProblem), cudaMemcpyHostToDevice, wk->stream));
  ProfScope ps(wk, 0, work, bytes);
  k_dyn_diag_grp<<<dim3((max_nbe + 127) / 128, 1, count), 128, 0, wk->stream>>>(dd);
  BEM_CUDA(wk, cudaGetLastError());
  k_dyn_offdiag_grp<<<dim3((max_nbe + kRowsPerCta - 1) / kRowsPerCta, max_chunks, count), 128, smem, wk->stream>>>(
      dd);
  BEM_CUDA(wk, cudaGetLastError());
  const int pb = (int)std::min<long long>((max_pad + 255) / 256, 256);
  k_rhs_pad_grp<<<dim3(pb, count), 256, 0, wk->stream>>>(dd);
  BEM_CUDA(wk, cudaGetLastError());
  wk->launches += 3;
  return BEM_OK;
}

// The per-frequency constants of a captured step: every k_dyn_diag and
// k_dyn_offdiag node of `exec` (listed in `nodes`) gets the parameters
// launch_dynamic_batch would pass for `b`; grids and shared memory stay.
int dyn_graph_update(bem_ctx* ctx, cudaGraphExec_t exec, const std::vector<cudaGraphNode_t>& nodes,
                     const DynBatch& b) {
  DynParams p = dyn_params(ctx, b);
  void* args[] = {&p};
  for (cudaGraphNode_t n : nodes) {
    cudaKernelNodeParams kp{};
    BEM_CUDA(ctx, cudaGraphKernelNodeGetParams(n, &kp));
    kp.kernelParams = args;
    kp.extra = nullptr;
    BEM_CUDA(ctx, cudaGraphExecKernelNodeSetParams(exec, n, &kp));
  }
  return BEM_OK;
}

// The dynamic-assembly kernel nodes of a captured graph.
int dyn_graph_nodes(bem_ctx* ctx, cudaGraph_t g, std::vector<cudaGraphNode_t>& out) {
  size_t n = 0;
  BEM_CUDA(ctx, cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> all(n);
  BEM_CUDA(ctx, cudaGraphGetNodes(g, all.data(), &n));
  out.clear();
  for (cudaGraphNode_t node : all) {
    cudaGraphNodeType t;
    BEM_CUDA(ctx, cudaGraphNodeGetType(node, &t));
    if (t != cudaGraphNodeTypeKernel) continue;
    cudaKernelNodeParams kp{};
    BEM_CUDA(ctx, cudaGraphKernelNodeGetParams(node, &kp));
    if (kp.func == (void*)k_dyn_diag || kp.func == (void*)k_dyn_offdiag) out.push_back(node);
  }
  return BEM_OK;
}

int launch_dynamic_batch(bem_ctx* ctx, const DynBatch& b) {
  Mesh& m = ctx->mesh;
  const int jc = jc_for(m.ng);
  const int chunks = (m.nbe + jc - 1) / jc;
  if (b.batch < 1 || b.batch > kMaxBatch) return fail(ctx, BEM_ERR_ARG, "batch size out of range");
  DynParams p = dyn_params(ctx, b);

  // work: Stokes evaluations; bytes: the FP64 system (and its complex64 copy) written once
  ProfScope ps(ctx, 0, (double)m.nbe * (double)m.nbe * (double)m.ng * b.batch,
               (double)(3 * m.nbe) * (3 * m.nbe + 1) * (16.0 + (b.A32 ? 8.0 : 0.0)) * b.batch);
  k_dyn_diag<<<dim3((m.nbe + 127) / 128, 1, b.batch), 128, 0, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  const size_t smem = (size_t)jc * m.ng * sizeof(double4);
  dim3 grid((m.nbe + kRowsPerCta - 1) / kRowsPerCta, chunks, b.batch);
  k_dyn_offdiag<<<grid, 128, smem, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  k_rhs_reduce<<<dim3((p.nn + 255) / 256, b.batch), 256, 0, ctx->stream>>>(p.nn, chunks, b.lda, b.a_stride,
                                                                           b.rhs_part, b.A, b.A32);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

int rhs_chunks(bem_ctx* ctx) {
  const int jc = jc_for(ctx->mesh.ng);
  return (ctx->mesh.nbe + jc - 1) / jc;
}

int launch_dynamic(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2],
                   const double c[4], double fr, int flags) {
  Mesh& m = ctx->mesh;
  System& s = ctx->sys;
  const int chunks = rhs_chunks(ctx);
  if (chunks > s.rhs_chunks) {
    if (s.rhs_part) dev_free(ctx, s.rhs_part);
    s.rhs_part = nullptr;
    BEM_CUDA(ctx, dev_alloc(ctx, &s.rhs_part, (size_t)chunks * s.nn * sizeof(double2)));
    s.rhs_chunks = chunks;
  }
  (void)m;
  DynBatch b{};
  b.zge = zge;
  b.zcs = zcs;
  b.zcp = zcp;
  b.c = c;
  b.freqs = &fr;
  b.batch = 1;
  b.flags = flags;
  b.A = s.A;
  b.lda = s.lda;
  b.a_stride = 0;
  b.A32 = nullptr;
  b.zh_pre = (flags & BEM_KEEP_PRESWAP) ? s.zh_pre : nullptr;
  b.zg_pre = (flags & BEM_KEEP_PRESWAP) ? s.zg_pre : nullptr;
  b.diag_h = s.diag_h;
  b.diag_g = s.diag_g;
  b.rhs_part = s.rhs_part;
  return launch_dynamic_batch(ctx, b);
}

// ---------------------------------------------------------------------------
// Static boundary system (an extension: the reference keeps only the static
// diagonals).  H(3I+i, 3J+j): Kelvin T of element J seen from collocation
// point I (SOLFUNE, Solfune.for:18-31, NPG^2 rule of Nonsinge.for), G: Kelvin
// U (SOLFUNE_G, Singge.for:195-198, rule of NONSINGE_G); I == J blocks are
// HESTdiag and GESTdiag.  Then the boundary-condition swap with the real GE
// (as Ghmatecd.for:316-333); A receives H (imaginary parts 0), Gs the
// post-swap G (real, nn x nn).  32 collocation rows per warp, one element
// column per warp iteration (coalesced column-major stores).
// ---------------------------------------------------------------------------
struct StaticSysParams {
  int nbe, nn, ng;
  size_t lda;
  double c1, c2, c3, c4, ge;
  const double4* gq;
  const double4* eta;
  const double4* colloc;
  const double* hestdiag;
  const double* gestdiag;
  const int* kode;
  double2* A;
  double* Gs;
};

__global__ void __launch_bounds__(128) k_static_system(StaticSysParams p) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int I = blockIdx.x * 32 + lane;
  if (I >= p.nbe) return;
  const double4 P = p.colloc[I];
  for (int J = blockIdx.y * 4 + w; J < p.nbe; J += gridDim.y * 4) {
    double T[3][3], U[3][3];
    if (J != I) {
      const double4 nv = p.eta[J];
      const double n3[3] = {nv.x, nv.y, nv.z};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) T[i][j] = U[i][j] = 0.0;
      const double4* q = p.gq + (size_t)J * p.ng;
      for (int g = 0; g < p.ng; ++g) {
        const double4 qq = q[g];
        const double r1 = qq.x - P.x, r2 = qq.y - P.y, r3 = qq.z - P.z;
        const double rr = fma(r1, r1, fma(r2, r2, r3 * r3));
        const double ir = rsqrt(rr);
        const double rd[3] = {r1 * ir, r2 * ir, r3 * ir};
        const double rdn = rd[0] * n3[0] + rd[1] * n3[1] + rd[2] * n3[2];
        const double ct = p.c3 * ir * ir * qq.w, cu = p.c1 * ir * qq.w;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const double dij = (i == j) ? 1.0 : 0.0;
            T[i][j] = fma(ct, rdn * (p.c4 * dij + 3.0 * rd[i] * rd[j]) + p.c4 * (rd[j] * n3[i] - rd[i] * n3[j]), T[i][j]);
            U[i][j] = fma(cu, p.c2 * dij + rd[i] * rd[j], U[i][j]);
          }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          T[i][j] = p.hestdiag[(size_t)9 * J + 3 * j + i];
          U[i][j] = p.gestdiag[(size_t)9 * J + 3 * j + i];
        }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int col = 3 * J + j;
      const bool swap = p.kode[col] == 0;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const size_t row = (size_t)3 * I + i;
        double h = T[i][j], g = U[i][j];
        if (swap) {
          const double hg = h * p.ge;
          h = -g;
          g = -hg;
        }
        p.A[(size_t)col * p.lda + row] = make_double2(h, 0.0);
        p.Gs[(size_t)col * p.nn + row] = g;
      }
    }
  }
}

// Right-hand side: column nn of A = Gs * dfi (one thread per row).
__global__ void k_static_rhs(const double* __restrict__ Gs, int nn, const double* __restrict__ dfi, double2* A,
                             size_t lda) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nn) return;
  double acc = 0.0;
  for (int c = 0; c < nn; ++c) acc = fma(Gs[(size_t)c * nn + r], dfi[c], acc);
  A[(size_t)nn * lda + r] = make_double2(acc, 0.0);
}

int launch_static_system(bem_ctx* ctx, const double c[4], double ge, const int* d_kode, const double* d_dfi,
                         double2* A, size_t lda, double* Gs) {
  const Mesh& m = ctx->mesh;
  StaticSysParams p{};
  p.nbe = m.nbe;
  p.nn = 3 * m.nbe;
  p.ng = m.ng;
  p.lda = lda;
  p.c1 = c[0];
  p.c2 = c[1];
  p.c3 = c[2];
  p.c4 = c[3];
  p.ge = ge;
  p.gq = m.gq;
  p.eta = m.eta;
  p.colloc = m.colloc;
  p.hestdiag = ctx->hestdiag;
  p.gestdiag = ctx->gestdiag;
  p.kode = d_kode;
  p.A = A;
  p.Gs = Gs;
  const int ycols = std::max(1, std::min((m.nbe + 3) / 4, 4 * ctx->num_sms * 4 / std::max(1, (m.nbe + 31) / 32)));
  k_static_system<<<dim3((m.nbe + 31) / 32, ycols), 128, 0, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  k_static_rhs<<<(p.nn + 127) / 128, 128, 0, ctx->stream>>>(Gs, p.nn, d_dfi, A, lda);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  return BEM_OK;
}

// ---------------------------------------------------------------------------
// GHMATECD without allocation (bem_ghmatecd_noalloc).
//
// The assembly needs two scratch buffers besides its inputs and outputs: the
// pre-swap diagonal blocks written by k_dyn_diag and read by k_dyn_offdiag
// (2 x 9 x nbe complex), and the per-chunk partial sums of the right-hand side
// written by k_dyn_offdiag and summed by k_rhs_reduce (chunks x 3nbe
// complex).  This variant takes both from one fixed array that every device
// holds from the moment the library's kernels are loaded on it until the
// process exits, so a call allocates nothing.  Every scratch word the kernels
// read is first written by the same call, so nothing in it needs to start at
// zero; the status words live in the context and are cleared per call.
// ---------------------------------------------------------------------------

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per device
static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double2)];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double2* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up on the
// first call per device.  On the host the array's name stands for a host-side
// shadow, never for device memory, so only this address goes to kernels.  The
// cached address belongs to the device's current context: after a
// cudaDeviceReset the module may load at another address, so the cache does
// not survive a reset (the header says so).
int noalloc_scratch(bem_ctx* ctx, double2** out) {
  if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices)
    return fail(ctx, BEM_ERR_ARG, "bem_ghmatecd_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[ctx->device]) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || !addr) return cuda_fail(ctx, e, "cudaGetSymbolAddress(no-allocation scratch)");
    g_noalloc_addr[ctx->device] = static_cast<double2*>(addr);
  }
  *out = g_noalloc_addr[ctx->device];
  return BEM_OK;
}

// Scratch layout in complex128 words: diagonal H blocks, diagonal G blocks,
// then the RHS partials starting on a 256-byte boundary.
size_t noalloc_part_offset(int nbe) { return ((size_t)18 * nbe + 15) & ~(size_t)15; }
size_t noalloc_words(int nbe, int chunks) { return noalloc_part_offset(nbe) + (size_t)chunks * 3 * nbe; }

}  // namespace

}  // namespace bem

using namespace bem;

int bem_ghmatecd_noalloc(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2],
                         const double c[4], double fr, int flags, double* a, size_t lda) {
  if (!ctx || !zge || !zcs || !zcp || !c || !a) return BEM_ERR_ARG;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (flags & ~BEM_FAST_SINGULAR)
    return fail(ctx, BEM_ERR_ARG, "bem_ghmatecd_noalloc: only BEM_FAST_SINGULAR is accepted");
  if (!ctx->have_mesh || !ctx->have_dyn) return fail(ctx, BEM_ERR_STATE, "bem_ghmatecd_noalloc needs mesh and BCs");
  if ((flags & BEM_FAST_SINGULAR) && (!ctx->have_hest || !ctx->have_gest))
    return fail(ctx, BEM_ERR_STATE, "bem_ghmatecd_noalloc needs HESTdiag and GESTdiag");
  const Mesh& m = ctx->mesh;
  if (m.ng * (int)sizeof(double4) > 1024 * 32) return fail(ctx, BEM_ERR_ARG, "Gauss rule too large");
  const int nn = 3 * m.nbe;
  if (lda < (size_t)nn) return fail(ctx, BEM_ERR_ARG, "bem_ghmatecd_noalloc: lda < 3*nbe");
  if (reinterpret_cast<uintptr_t>(a) % alignof(double2) != 0)
    return fail(ctx, BEM_ERR_ARG, "bem_ghmatecd_noalloc: a must be 16-byte aligned");
  const int jc = jc_for(m.ng);
  const int chunks = (m.nbe + jc - 1) / jc;
  const size_t need = noalloc_words(m.nbe, chunks) * sizeof(double2);
  if (need > kNoAllocScratchBytes) {
    char msg[200];
    std::snprintf(msg, sizeof msg,
                  "bem_ghmatecd_noalloc: this mesh needs %zu bytes of scratch, the fixed limit is %zu bytes; "
                  "use bem_ghmatecd",
                  need, kNoAllocScratchBytes);
    return fail(ctx, BEM_ERR_ARG, msg);
  }
  BEM_CUDA(ctx, cudaSetDevice(ctx->device));
  double2* scratch = nullptr;
  int rc = noalloc_scratch(ctx, &scratch);
  if (rc) return rc;
  BEM_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream));

  DynParams p{};
  p.nbe = m.nbe;
  p.nn = nn;
  p.ng = m.ng;
  p.jc = jc;
  p.chunks = chunks;
  p.lda = lda;
  p.a_stride = 0;
  p.zge = make_double2(zge[0], zge[1]);
  p.c1 = c[0];
  p.c2 = c[1];
  p.c3 = c[2];
  p.c4 = c[3];
  p.fast_singular = (flags & BEM_FAST_SINGULAR) ? 1 : 0;
  p.gq = m.gq;
  p.eta = m.eta;
  p.colloc = m.colloc;
  p.hestdiag = ctx->hestdiag;
  p.gestdiag = ctx->gestdiag;
  p.kode = ctx->kode;
  p.zdfi = ctx->zdfi;
  p.A = reinterpret_cast<double2*>(a);
  p.A32 = nullptr;
  p.zh_pre = nullptr;
  p.zg_pre = nullptr;
  p.diag_h = scratch;
  p.diag_g = scratch + (size_t)9 * m.nbe;
  p.rhs_part = scratch + noalloc_part_offset(m.nbe);
  p.status = ctx->d_status;
  p.kb[0] = make_consts(zge, zcs, zcp, fr);

  // timed as the assembly class when profiling is on, like bem_ghmatecd:
  // work = Stokes evaluations, bytes = the system written once
  ProfScope ps(ctx, 0, (double)m.nbe * (double)m.nbe * (double)m.ng, (double)nn * (nn + 1) * 16.0);
  k_dyn_diag<<<dim3((m.nbe + 127) / 128, 1, 1), 128, 0, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  const size_t smem = (size_t)jc * m.ng * sizeof(double4);
  k_dyn_offdiag<<<dim3((m.nbe + kRowsPerCta - 1) / kRowsPerCta, chunks, 1), 128, smem, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  k_rhs_reduce<<<dim3((nn + 255) / 256, 1), 256, 0, ctx->stream>>>(nn, chunks, lda, 0, p.rhs_part, p.A, nullptr);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  if (ctx->mesh_flag_bnd) return fail(ctx, BEM_ERR_DEGENERATE, "Jacobian below 1e-5 on a boundary element");
  return BEM_OK;
}
