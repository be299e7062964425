// interior.cu -- displacements and stresses at interior points on the device.
//
// INTEREC's interior part: the displacement at interior point K is
//   ZDSOL(3K+i) = sum_J  ZG_KJ(i,:) . ZDFI_J  -  ZH_KJ(i,:) . ZFI_J
// with NONSINGD's Stokes U and T over boundary element J seen from K
// (src/Interec.for:86-135, the computation cuda_interec1_ does on the
// reference's GPU, src/kernels/Interec1_cu.cu:44-237), and the stress is
//   ZSSOL(9K+i+3j) = sum_J sum_k ZDFI_J(k) ZD(k,i,j) - ZFI_J(k) ZS(k,i,j)
// with SIGMAEC's derivative kernels (src/Interec.for:186-285,
// src/Sigmaec.for:9-212).  ZFI / ZDFI are the boundary displacements and
// tractions after the un-swap.
//
// One thread per (interior point, boundary element): the NPG^2 Gauss points
// of the element (the per-mesh table of k_geometry) are visited once, and at
// every Gauss point U, T, ZD and ZS are contracted with the element's
// tractions and displacements straight away (algebraically the reference's
// sum of element matrices times the boundary vectors; ZD and ZS contract to
// tensors symmetric in (i, j), so 6 stress components are accumulated).  A
// CTA reduces its 128 elements in a fixed order and writes one partial per
// (point, element chunk); k_interior_reduce sums the chunks in order, so the
// result does not depend on scheduling.
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <vector>

#include "bem_internal.h"

namespace bem {

namespace {

constexpr int kIntThreads = 128;  // boundary elements per CTA, one per thread
constexpr int kIntOut = 12;       // 3 displacement + 9 stress components
constexpr int kIntAcc = 9;        // 3 displacement + 6 symmetric stress components

struct InteriorParams {
  int nbe, ng, l, chunks, want_stress;
  const double4* gq;   // [N][ng] Gauss point (x, y, z, w1*w2*|J|)
  const double4* eta;  // [N] unit normals
  const double4* pts;  // [l] interior points
  const double2* u;    // [3nbe] boundary displacements
  const double2* t;    // [3nbe] boundary tractions
  StokesConsts<double> kc;
  zd zmu, lm;          // shear modulus ZGE, and lambda / mu
  double2* part;       // [l][chunks][12]
};

__device__ __forceinline__ zd ldz(const double2* p) {
  const double2 v = *p;
  return zd{v.x, v.y};
}

// Symmetric index (i <= j) -> 0..5: 00 01 02 11 12 22.
__host__ __device__ constexpr int sidx(int i, int j) {
  return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5)) : (j == 0 ? i : (j == 1 ? 2 + i : 5));
}

__global__ void __launch_bounds__(kIntThreads) k_interior(InteriorParams p) {
  __shared__ zd s_red[kIntThreads / 32][kIntAcc];
  const int K = blockIdx.y;
  const int J = blockIdx.x * kIntThreads + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  zd acc[kIntAcc];
#pragma unroll
  for (int i = 0; i < kIntAcc; ++i) acc[i] = zd{0.0, 0.0};

  if (J < p.nbe) {
    const StokesConsts<double>& kc = p.kc;
    const double4 P = p.pts[K];
    const double4 nv = p.eta[J];
    const double n[3] = {nv.x, nv.y, nv.z};
    zd u[3], t[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      u[i] = ldz(&p.u[3 * J + i]);
      t[i] = ldz(&p.t[3 * J + i]);
    }
    zd un{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 3; ++i) cfma(un, u[i], n[i]);
    const double4* q = p.gq + (size_t)J * p.ng;
    for (int g = 0; g < p.ng; ++g) {
      const double4 qq = q[g];
      const double r1 = qq.x - P.x, r2 = qq.y - P.y, r3 = qq.z - P.z;
      const double rr = fma(r1, r1, fma(r2, r2, r3 * r3));
      const double ir = rsqrt(rr);  // r and 1/r from one rsqrt
      const double r = rr * ir;
      const double rd[3] = {r1 * ir, r2 * ir, r3 * ir};
      const double drn = rd[0] * n[0] + rd[1] * n[1] + rd[2] * n[2];
      const double wt = qq.w;
      // Radial functions, Solfund.for:36-49 (as stokes_radial) and the
      // second derivatives of Sigmaec.for, with zzs = -k2 r, zzp = -k1 r.
      const zd zzs = kc.zks * r, zzp = kc.zkp * r;
      const zd es = cexp_scaled(zzs, ir);           // exp(zzs) / r
      const zd ep = cexp_scaled(zzp, ir) * kc.zc2;  // (cs/cp)^2 exp(zzp) / r
      const zd izs = kc.izks * ir, izp = kc.izkp * ir;
      const zd izs2 = izs * izs, izp2 = izp * izp;
      const zd fhi = (1.0 + izs2 - izs) * es - (izp2 - izp) * ep;
      const zd cappa = (1.0 + 3.0 * izs2 - 3.0 * izs) * es - (1.0 + 3.0 * izp2 - 3.0 * izp) * ep;
      const zd fhidr = ((-2.0 + zzs + 3.0 * izs - 3.0 * izs2) * es - (-1.0 + 3.0 * izp - 3.0 * izp2) * ep) * ir;
      const zd cappadr = ((zzs - 4.0 + 9.0 * izs - 9.0 * izs2) * es - (zzp - 4.0 + 9.0 * izp - 9.0 * izp2) * ep) * ir;
      const zd cr = cappa * ir;
      const zd aa = fhidr - cr;
      const zd bb = 4.0 * cr - 2.0 * cappadr;
      const zd cc = kc.zc1m2 * (aa + 0.5 * bb - 3.0 * cr) - 2.0 * cr;
      zd rt{0.0, 0.0}, ru{0.0, 0.0};
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        cfma(rt, t[i], rd[i]);
        cfma(ru, u[i], rd[i]);
      }
      // Displacements: U(i,:) . t - T(i,:) . u   (Solfund.for:50-60 layouts)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const zd ug = kc.zc0 * (fhi * t[i] - cappa * (rd[i] * rt));
        const zd th = kc.inv4pi * (aa * (drn * u[i] + n[i] * ru) + bb * (rd[i] * drn * ru) + cc * (rd[i] * un));
        cfma(acc[i], ug - th, wt);
      }
      if (p.want_stress) {
        const double ir2 = ir * ir;
        const zd zs2 = zzs * zzs, zp2 = zzp * zzp;
        const zd fhidrr = ((12.0 * izs2 - 12.0 * izs + 7.0 - 3.0 * zzs + zs2) * es -
                           (12.0 * izp2 - 12.0 * izp + 5.0 - zzp) * ep) * ir2;
        const zd cappadrr = ((36.0 * izs2 - 36.0 * izs + 17.0 - 5.0 * zzs + zs2) * es -
                             (36.0 * izp2 - 36.0 * izp + 17.0 - 5.0 * zzp + zp2) * ep) * ir2;
        const zd lm = p.lm;
        const zd cr2 = cappa * ir2, fr1 = fhidr * ir, cr1 = cappadr * ir;
        const zd c1 = 2.0 * cr;
        const zd c2 = lm * (fhidr - cappadr - c1);
        const zd c3 = fhidr - cr;
        const zd c4 = 2.0 * (cappadr - c1);
        const zd c5 = 4.0 * (cappadrr - 5.0 * cr1 + 8.0 * cr2);
        const zd c6 = fhidrr - fr1 - 3.0 * cr1 + 6.0 * cr2;
        const zd c7 = 2.0 * cr1 - 4.0 * cr2;
        const zd c8 = lm * (cappadrr + cr1 - 4.0 * cr2 - fhidrr + fr1);
        const zd c9 = 2.0 * (c7 + c8);
        const zd c10 = 4.0 * cr2 + 4.0 * lm * (cr1 + 2.0 * cr2 - fr1);
        const zd c11 = (lm * lm) * (cappadrr + 4.0 * cr1 + 2.0 * cr2 - fhidrr - 2.0 * fr1);
        const zd c12 = 2.0 * (fr1 - cr2);
        const zd c12a = c1 - c2, c1011 = c10 + c11;
        const zd mu4 = p.zmu * kc.inv4pi;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = i; j < 3; ++j) {
            const double rij = rd[i] * rd[j];
            // sum_k t_k ZD(k,i,j)
            zd d = c4 * (rij * rt) - c3 * (t[j] * rd[i] + t[i] * rd[j]);
            if (i == j) d = d + c12a * rt;
            d = kc.inv4pi * d;
            // sum_k u_k ZS(k,i,j)
            zd s = drn * (c5 * (rij * ru) - c6 * (u[j] * rd[i] + u[i] * rd[j])) + c9 * (rij * un) -
                   c6 * ((rd[i] * n[j] + rd[j] * n[i]) * ru) - c12 * (u[i] * n[j] + u[j] * n[i]);
            if (i == j) s = s + c9 * (drn * ru) + c1011 * un;
            s = mu4 * s;
            cfma(acc[3 + sidx(i, j)], d - s, wt);
          }
      }
    }
  }
  // CTA reduction in a fixed order: warp tree, then the 4 warps in order.
#pragma unroll
  for (int i = 0; i < kIntAcc; ++i) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc[i].re += __shfl_down_sync(0xffffffffu, acc[i].re, off);
      acc[i].im += __shfl_down_sync(0xffffffffu, acc[i].im, off);
    }
    if (lane == 0) s_red[warp][i] = acc[i];
  }
  __syncthreads();
  if (threadIdx.x < kIntOut) {
    const int o = threadIdx.x;
    // output o: 0..2 displacement, 3 + (i + 3j) stress component (i, j)
    const int a = o < 3 ? o : 3 + sidx((o - 3) % 3, (o - 3) / 3);
    zd sum = s_red[0][a];
#pragma unroll
    for (int w = 1; w < kIntThreads / 32; ++w) sum = sum + s_red[w][a];
    p.part[((size_t)K * p.chunks + blockIdx.x) * kIntOut + o] = make_double2(sum.re, sum.im);
  }
}

__global__ void k_interior_reduce(const double2* __restrict__ part, int l, int chunks, double2* out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= l * kIntOut) return;
  const int K = idx / kIntOut, o = idx % kIntOut;
  double2 s = make_double2(0.0, 0.0);
  for (int c = 0; c < chunks; ++c) {
    const double2 v = part[((size_t)K * chunks + c) * kIntOut + o];
    s.x += v.x;
    s.y += v.y;
  }
  out[idx] = s;
}

}  // namespace

void release_interior(bem_ctx* ctx) {
  dev_free(ctx, ctx->int_pts);
  dev_free(ctx, ctx->int_ut);
  dev_free(ctx, ctx->int_part);
  dev_free(ctx, ctx->int_out);
  ctx->int_pts = nullptr;
  ctx->int_ut = nullptr;
  ctx->int_part = nullptr;
  ctx->int_out = nullptr;
  ctx->int_cap_l = ctx->int_cap_nn = 0;
}

int interior_points(bem_ctx* ctx, const double zge[2], const double zcs[2], const double zcp[2], double rho,
                    double fr, int l, const double* cxi, const double* cyi, const double* czi, const double* disp,
                    const double* trac, double* zdsol, double* zssol) {
  const Mesh& m = ctx->mesh;
  const int nbe = m.nbe, nn = 3 * nbe;
  if (l <= 0) return BEM_OK;
  const int chunks = (nbe + kIntThreads - 1) / kIntThreads;
  if ((size_t)l > ctx->int_cap_l || (size_t)nn > ctx->int_cap_nn) {
    release_interior(ctx);
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->int_pts, (size_t)l * sizeof(double4)));
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->int_ut, (size_t)2 * nn * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->int_part, (size_t)l * chunks * kIntOut * sizeof(double2)));
    BEM_CUDA(ctx, dev_alloc(ctx, &ctx->int_out, (size_t)l * kIntOut * sizeof(double2)));
    ctx->int_cap_l = (size_t)l;
    ctx->int_cap_nn = (size_t)nn;
  }
  std::vector<double4> pts((size_t)l);
  for (int k = 0; k < l; ++k) pts[k] = make_double4(cxi[k], cyi[k], czi[k], 0.0);
  BEM_CUDA(ctx, cudaMemcpyAsync(ctx->int_pts, pts.data(), (size_t)l * sizeof(double4), cudaMemcpyHostToDevice,
                                ctx->stream));
  BEM_CUDA(ctx, cudaMemcpyAsync(ctx->int_ut, disp, (size_t)nn * sizeof(double2), cudaMemcpyHostToDevice,
                                ctx->stream));
  BEM_CUDA(ctx, cudaMemcpyAsync(ctx->int_ut + nn, trac, (size_t)nn * sizeof(double2), cudaMemcpyHostToDevice,
                                ctx->stream));
  using cd = std::complex<double>;
  const cd zmu(zge[0], zge[1]), cp(zcp[0], zcp[1]);
  const cd lm = (cp * cp * rho - 2.0 * zmu) / zmu;  // Sigmaec.for: ZLAMB / ZMU
  InteriorParams p{};
  p.nbe = nbe;
  p.ng = m.ng;
  p.l = l;
  p.chunks = chunks;
  p.want_stress = zssol ? 1 : 0;
  p.gq = m.gq;
  p.eta = m.eta;
  p.pts = ctx->int_pts;
  p.u = ctx->int_ut;
  p.t = ctx->int_ut + nn;
  p.kc = make_consts(zge, zcs, zcp, fr);
  p.zmu = zd{zmu.real(), zmu.imag()};
  p.lm = zd{lm.real(), lm.imag()};
  p.part = ctx->int_part;
  k_interior<<<dim3(chunks, l), kIntThreads, 0, ctx->stream>>>(p);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  k_interior_reduce<<<(l * kIntOut + 255) / 256, 256, 0, ctx->stream>>>(ctx->int_part, l, chunks, ctx->int_out);
  ctx->launches++;
  BEM_CUDA(ctx, cudaGetLastError());
  std::vector<double2> out((size_t)l * kIntOut);
  BEM_CUDA(ctx, cudaMemcpyAsync(out.data(), ctx->int_out, out.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                                ctx->stream));
  BEM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < l; ++k) {
    for (int i = 0; i < 3; ++i) {
      zdsol[2 * (3 * k + i)] = out[(size_t)k * kIntOut + i].x;
      zdsol[2 * (3 * k + i) + 1] = out[(size_t)k * kIntOut + i].y;
    }
    if (zssol)
      for (int mm = 0; mm < 9; ++mm) {
        zssol[2 * (9 * k + mm)] = out[(size_t)k * kIntOut + 3 + mm].x;
        zssol[2 * (9 * k + mm) + 1] = out[(size_t)k * kIntOut + 3 + mm].y;
      }
  }
  return BEM_OK;
}

}  // namespace bem
