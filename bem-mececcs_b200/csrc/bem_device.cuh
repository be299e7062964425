// bem_device.cuh -- device helpers shared by the assembly and LU kernels.
//
// Complex numbers are plain (re, im) pairs, the layout of Fortran COMPLEX*16
// and of the reference's thrust::complex<double> (src/kernels/shared.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bem {

// Status words in device memory (ctx->d_status[]).
enum DevStatus { ST_DEGENERATE = 0, ST_SINGULAR = 1, ST_TIMEOUT = 2, ST_COUNT = 4 };
// After the status words: two mesh flags (ints 4, 5), the context's wait
// limit (a u64 of nanoseconds at ints 6-7, 8-byte aligned; 0 = the default)
// and the counter of the wait self-test's grid barrier (int 8).
constexpr int ST_WAIT_LIMIT = 6;
constexpr int ST_SELFTEST_CTR = 8;
constexpr int ST_WORDS = 16;  // ints of ctx->d_status

// Bounded device waits give up after this many nanoseconds of %globaltimer
// unless the context sets its own limit (option "wait_limit_ms").
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

// The wait limit of the context that owns `status`; read once per kernel.
__device__ __forceinline__ unsigned long long wait_limit(const int* status) {
  const unsigned long long v =
      status ? *reinterpret_cast<const volatile unsigned long long*>(status + ST_WAIT_LIMIT) : 0ull;
  return v ? v : kWaitLimitNs;
}

template <typename R>
struct cpx {
  R re, im;
};
using zd = cpx<double>;
using zf = cpx<float>;

template <typename R>
__device__ __forceinline__ cpx<R> mk(R a, R b) { return cpx<R>{a, b}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return {a.re - b.re, a.im - b.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator-(cpx<R> a) { return {-a.re, -a.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator*(cpx<R> a, cpx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename R>
__device__ __forceinline__ cpx<R> operator*(cpx<R> a, R s) { return {a.re * s, a.im * s}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator*(R s, cpx<R> a) { return {a.re * s, a.im * s}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator+(cpx<R> a, R s) { return {a.re + s, a.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator+(R s, cpx<R> a) { return {a.re + s, a.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator-(cpx<R> a, R s) { return {a.re - s, a.im}; }
template <typename R>
__device__ __forceinline__ cpx<R> operator-(R s, cpx<R> a) { return {s - a.re, -a.im}; }
// a += b * c
template <typename R>
__device__ __forceinline__ void cfma(cpx<R>& a, cpx<R> b, cpx<R> c) {
  a.re = fma(b.re, c.re, fma(-b.im, c.im, a.re));
  a.im = fma(b.re, c.im, fma(b.im, c.re, a.im));
}
// a += b * s (s real)
template <typename R>
__device__ __forceinline__ void cfma(cpx<R>& a, cpx<R> b, R s) {
  a.re = fma(b.re, s, a.re);
  a.im = fma(b.im, s, a.im);
}
// 1 / z, as conj(z) / |z|^2.
__device__ __forceinline__ zd crcp(zd z) {
  double s = 1.0 / fma(z.re, z.re, z.im * z.im);
  return {z.re * s, -z.im * s};
}
__device__ __forceinline__ zf crcp(zf z) {
  float s = __frcp_rn(fmaf(z.re, z.re, z.im * z.im));
  return {z.re * s, -z.im * s};
}
// exp(z) * scale.
__device__ __forceinline__ zd cexp_scaled(zd z, double scale) {
  double s, c;
  sincos(z.im, &s, &c);
  double e = exp(z.re) * scale;
  return {e * c, e * s};
}
__device__ __forceinline__ zf cexp_scaled(zf z, float scale) {
  float s, c;
  sincosf(z.im, &s, &c);
  float e = expf(z.re) * scale;
  return {e * c, e * s};
}
__device__ __forceinline__ double cabs1(zd z) { return fabs(z.re) + fabs(z.im); }
__device__ __forceinline__ float cabs1(zf z) { return fabsf(z.re) + fabsf(z.im); }

// Frequency constants of the Stokes solution, Solfund.for:29-35.
template <typename R>
struct StokesConsts {
  cpx<R> zkp, zks;   // -i w / cp, -i w / cs
  cpx<R> zc2;        // (cs/cp)^2
  cpx<R> zc1m2;      // (cp/cs)^2 - 2
  cpx<R> zc0;        // 1 / (4 pi zge)
  R inv4pi;
  cpx<R> izkp, izks; // 1 / zkp, 1 / zks: 1 / (zk r) = (1 / zk) (1 / r), no division per point
};

// The radial functions of the Stokes solution at distance r (inverse ir),
// Solfund.for:36-49: returns FHI, CAPPA, AA, BB, CC.
template <typename R>
struct StokesRadial {
  cpx<R> fhi, cappa, aa, bb, cc;
};

template <typename R>
__device__ __forceinline__ StokesRadial<R> stokes_radial(const StokesConsts<R>& k, R r, R ir) {
  cpx<R> zzs = k.zks * r, zzp = k.zkp * r;
  cpx<R> es = cexp_scaled(zzs, ir);           // exp(zzs) / r
  cpx<R> ep = cexp_scaled(zzp, ir) * k.zc2;   // zc2 exp(zzp) / r
  cpx<R> izs = k.izks * ir, izp = k.izkp * ir;
  cpx<R> izs2 = izs * izs, izp2 = izp * izp;
  const R one = R(1), two = R(2), three = R(3), four = R(4), nine = R(9);
  StokesRadial<R> s;
  s.fhi = (one + izs2 - izs) * es - (izp2 - izp) * ep;
  s.cappa = (one + three * izs2 - three * izs) * es - (one + three * izp2 - three * izp) * ep;
  cpx<R> fhidr = ((-two + zzs + three * izs - three * izs2) * es -
                  (-one + three * izp - three * izp2) * ep) * ir;
  cpx<R> cappadr = ((zzs - four + nine * izs - nine * izs2) * es -
                    (zzp - four + nine * izp - nine * izp2) * ep) * ir;
  cpx<R> cr = s.cappa * ir;
  s.aa = fhidr - cr;
  s.bb = four * cr - two * cappadr;
  s.cc = k.zc1m2 * (s.aa + R(0.5) * s.bb - three * cr) - two * cr;
  return s;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of a cooperative launch over `nblocks` CTAs.  `ctr` is
// zeroed before the launch; barrier number `epoch` (1, 2, ...) completes when
// the counter reaches epoch * nblocks.  The wait is bounded by limit_ns (the
// context's wait_limit): on timeout (or when another CTA has already timed
// out) it sets status[ST_TIMEOUT] and returns false; callers then leave the
// kernel.
__device__ __forceinline__ bool grid_barrier(unsigned* ctr, unsigned epoch, unsigned nblocks,
                                             int* status, unsigned long long limit_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    red_release_gpu_add(ctr, 1u);
    const unsigned target = epoch * nblocks;
    const unsigned long long t0 = globaltimer_ns();
    int ok = 1;
    unsigned spins = 0;
    while (ld_acquire_gpu(ctr) < target) {
      if ((++spins & 255u) == 0) {
        if (*(volatile int*)&status[ST_TIMEOUT] != 0 || globaltimer_ns() - t0 > limit_ns) {
          atomicExch(&status[ST_TIMEOUT], 1);
          ok = 0;
          break;
        }
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// ---- 1-D bulk copy (TMA engine) global -> shared with an mbarrier. ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bytes must be a multiple of 16; both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait for phase `parity` of the mbarrier; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned long long limit_ns = kWaitLimitNs) {
  // the clock is read only once the first try has failed: a wait that is
  // already satisfied (the common case in a full pipeline) costs one try
  unsigned long long t0 = 0;
  unsigned spins = 0;
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (spins == 0) t0 = globaltimer_ns();
    if ((++spins & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) return false;
  }
}

}  // namespace bem
