// serve.cu -- the serving form: a request loop over resident meshes.
//
// Requests (mesh, material, omega, boundary conditions) arrive through
// bem_server_submit and are solved as they come: a scheduler thread admits
// every request that fits the HBM budget into a slot -- one context (own
// stream, own workspaces) holding one problem -- and enqueues its work
// asynchronously, so requests that arrive while others are on the GPU run
// concurrently with them on the device (continuous batching over streams).
// After a solve the slot keeps the problem resident: the FP64 H, its
// factors and the post-swap G.  A later request for the same (mesh,
// material, omega, KODE) with a new right-hand side is then a GEMV plus the
// cached solve (RHS-only).  Admission is by the slot's device footprint
// (about 2 n^2 complex128 entries: H and G, plus the complex64 factors in the
// mixed form); idle slots are evicted least-recently-used to make room.
// Completion is observed with one CUDA event per slot; results land in
// pinned host buffers, so the loop never blocks on a copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bem_internal.h"

namespace bem {
namespace {

using Clock = std::chrono::steady_clock;

// Work in flight at once: at most 8 slots (independent solves or lockstep
// batches) and 16 problems.  Every LU keeps one panel cluster per problem and
// the device holds about 9 16-CTA clusters at a time; admitting more than
// that only queues kernels behind each other (measured: 94 concurrent
// 6480-unknown solves ran 4x slower in total than 16), so a request that fits
// the memory budget still waits here until a solve finishes.  16 problems let
// two lockstep batches of a sweep run side by side, one's panels overlapping
// the other's updates.
constexpr int kMaxInflight = 16;
constexpr int kMaxSlotsBusy = 8;
constexpr int kDefer = -2;  // try_start: wait for a fuller lockstep batch
// A request waits for a fuller batch at most this long after its submission,
// so that a busy server cannot starve it (it then starts with what fits).
constexpr double kDeferLimitMs = 1000.0;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct SrvMesh {
  int n = 0, nbe = 0, np = 0, npg = 0;
  std::vector<int> cone;
  std::vector<double> cx, cy, cz, cxm, cym, czm, etas, gi, ome;
};

struct SrvRequest {
  long long id = 0;
  int mesh = 0;
  double mat[4] = {0, 0, 0, 0};  // GE, nu, damping, density
  double fr = 0.0;
  std::vector<double> bc;  // 3 nbe complex
  std::vector<int> kode;   // 3 nbe
  Clock::time_point t_submit, t_start, t_done;
  long long pkey = 0;  // problem key: equal for equal (mesh, material, BCs, KODE)
  bool started = false, done = false, rhs_only = false;
  int status = BEM_OK;
  size_t bytes = 0;
  std::vector<double> disp, trac;  // results after the un-swap
};

struct Slot {
  bem_ctx* ctx = nullptr;
  int mesh = -1;
  bool busy = false, cached = false;
  double mat[4] = {0, 0, 0, 0};
  double fr = 0.0;
  std::vector<int> kode;
  bool have_static = false;
  double st_ge = 0.0, st_nu = 0.0;
  size_t bytes = 0;
  unsigned long long last_use = 0;
  cudaEvent_t done = nullptr;
  double* h_x = nullptr;  // pinned, 2 nn doubles per problem (h_cap bytes)
  size_t h_cap = 0;
  int cap_probs = 1;      // problems the slot's bytes were admitted for
  std::vector<std::shared_ptr<SrvRequest>> reqs;  // in flight: one, or a lockstep batch
};

// Inputecd.for:58-60 and Ghmatece.for:55-63 on the host.
void material_consts(const double mat[4], double zge[2], double zcs[2], double zcp[2]) {
  using cd = std::complex<double>;
  const double ge = mat[0], nu = mat[1], dam = mat[2], rho = mat[3];
  const cd g = cd(ge, 0.0) * cd(1.0, 2.0 * dam);
  const cd cs = std::sqrt(g / rho);
  const cd cp = cs * std::sqrt((2.0 - 2.0 * nu) / (1.0 - 2.0 * nu));
  zge[0] = g.real(), zge[1] = g.imag();
  zcs[0] = cs.real(), zcs[1] = cs.imag();
  zcp[0] = cp.real(), zcp[1] = cp.imag();
}

void static_consts(double ge, double nu, double c[4]) {
  const double pi = 4.0 * std::atan(1.0);
  c[0] = 1.0 / (16.0 * pi * ge * (1.0 - nu));
  c[1] = 3.0 - 4.0 * nu;
  c[2] = -1.0 / (8.0 * pi * (1.0 - nu));
  c[3] = 1.0 - 2.0 * nu;
}

}  // namespace

class Server {
 public:
  Server(int device, double budget, int form, int refine)
      : device_(device), budget_((size_t)budget), mixed_(form == BEM_FORM_MIXED), refine_(refine) {
    worker_ = std::thread([this] { loop(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    worker_.join();
    cudaSetDevice(device_);
    for (Slot& s : slots_) destroy_slot(s);
    if (probe_) bem_ctx_destroy(probe_);
    for (auto& b : pinned_free_) cudaFreeHost(b.second);
    // hand the device memory the slots held back from the stream-ordered pool
    cudaMemPool_t pool;
    if (cudaDeviceSynchronize() == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
  }

  int add_mesh(SrvMesh&& m) {
    std::lock_guard<std::mutex> lk(mu_);
    meshes_.push_back(std::move(m));
    return (int)meshes_.size() - 1;
  }

  int submit(int mesh, const double mat[4], double fr, const double* bc, const int* kode, long long* id) {
    std::lock_guard<std::mutex> lk(mu_);
    if (mesh < 0 || mesh >= (int)meshes_.size()) return BEM_ERR_ARG;
    const int nn = 3 * meshes_[mesh].nbe;
    auto r = std::make_shared<SrvRequest>();
    r->id = ++next_id_;
    r->mesh = mesh;
    std::memcpy(r->mat, mat, sizeof r->mat);
    r->fr = fr;
    r->bc.assign(bc, bc + 2 * (size_t)nn);
    r->kode.assign(kode, kode + nn);
    r->pkey = problem_key(r);
    r->t_submit = Clock::now();
    if (!have_first_) {
      first_submit_ = r->t_submit;
      have_first_ = true;
    }
    reqs_[r->id] = r;
    queue_.push_back(r);
    *id = r->id;
    cv_.notify_all();
    return BEM_OK;
  }

  int wait(long long id, double timeout_s, double* disp, double* trac, double* info) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return BEM_ERR_ARG;
    std::shared_ptr<SrvRequest> r = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    if (!done_cv_.wait_until(lk, until, [&] { return r->done; })) return BEM_ERR_TIMEOUT;
    const size_t nn = r->kode.size();
    if (r->status == BEM_OK) {
      if (disp) std::memcpy(disp, r->disp.data(), 2 * nn * sizeof(double));
      if (trac) std::memcpy(trac, r->trac.data(), 2 * nn * sizeof(double));
    }
    if (info) {
      info[0] = ms_between(r->t_submit, r->t_done);
      info[1] = r->started ? ms_between(r->t_submit, r->t_start) : 0.0;
      info[2] = r->rhs_only ? 1.0 : 0.0;
      info[3] = (double)r->bytes;
    }
    const int st = r->status;
    reqs_.erase(it);
    return st;
  }

  void stats(double* out) {
    std::lock_guard<std::mutex> lk(mu_);
    std::vector<double> l = lat_;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
      if (l.empty()) return 0.0;
      const size_t i = (size_t)std::min<double>(l.size() - 1, std::ceil(q * l.size()) - 1);
      return l[i];
    };
    out[0] = (double)l.size();
    out[1] = pct(0.50);
    out[2] = pct(0.99);
    out[3] = (have_first_ && !l.empty()) ? l.size() / (ms_between(first_submit_, last_done_) * 1e-3) : 0.0;
    out[4] = (double)n_rhs_only_;
    out[5] = (double)n_evict_;
    out[6] = (double)peak_bytes_;
    out[7] = (double)max_busy_;
    out[8] = (double)used_bytes_;
    out[9] = (double)budget_;
  }

  void reset_stats() {
    std::lock_guard<std::mutex> lk(mu_);
    lat_.clear();
    n_rhs_only_ = n_evict_ = 0;
    peak_bytes_ = used_bytes_;
    max_busy_ = 0;
    have_first_ = false;
  }

 private:
  void loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    while (!stop_) {
      bool progress = false;
      int busy = 0, busy_slots = 0;  // problems and slots in flight
      for (Slot& s : slots_)
        if (s.busy) {
          if (cudaEventQuery(s.done) == cudaSuccess) {
            finish(s);
            progress = true;
          } else {
            busy += (int)s.reqs.size();
            ++busy_slots;
          }
        }
      for (auto it = queue_.begin(); it != queue_.end() && busy < kMaxInflight && busy_slots < kMaxSlotsBusy;) {
        const int st = try_start(*it, kMaxInflight - busy);
        if (st > 0) {  // the request and any batched with it leave the queue
          ++busy_slots;
          queue_.erase(std::remove_if(queue_.begin(), queue_.end(),
                                      [](const std::shared_ptr<SrvRequest>& q) { return q->started; }),
                       queue_.end());
          it = queue_.begin();
          progress = true;
          busy += st;
        } else if (st == kDefer) {
          ++it;  // waits for a fuller lockstep batch; later requests may start
        } else if (st < 0) {
          it = queue_.erase(it);  // failed at admission: reported through wait()
          progress = true;
        } else {
          ++it;
        }
      }
      max_busy_ = std::max(max_busy_, busy);
      if (!progress) cv_.wait_for(lk, std::chrono::microseconds(200));
    }
  }

  void complete(const std::shared_ptr<SrvRequest>& r, int status) {
    r->status = status;
    r->t_done = Clock::now();
    r->done = true;
    if (status == BEM_OK) {
      lat_.push_back(ms_between(r->t_submit, r->t_done));
      last_done_ = r->t_done;
      if (r->rhs_only) ++n_rhs_only_;
    }
    done_cv_.notify_all();
  }

  void finish(Slot& s) {
    std::vector<std::shared_ptr<SrvRequest>> rs;
    rs.swap(s.reqs);
    s.busy = false;
    int st;
    {
      std::lock_guard<std::mutex> g(s.ctx->mu);
      st = check_status(s.ctx);
    }
    if (st == BEM_OK && s.ctx->mesh_flag_bnd) st = BEM_ERR_DEGENERATE;
    s.cached = (st == BEM_OK && rs.size() == 1);  // a batch's problems are not kept for reuse
    s.last_use = ++tick_;
    for (size_t b = 0; b < rs.size(); ++b) finish_one(rs[b], st, s.h_x + 2 * rs[b]->kode.size() * b);
  }

  void finish_one(const std::shared_ptr<SrvRequest>& r, int st, const double* hx) {
    if (st == BEM_OK) {
      // The un-swap of Interec.for:59-67: KODE = 0 entries exchange roles.
      double zge[2], zcs[2], zcp[2];
      material_consts(r->mat, zge, zcs, zcp);
      const size_t nn = r->kode.size();
      r->disp.resize(2 * nn);
      r->trac.resize(2 * nn);
      for (size_t i = 0; i < nn; ++i) {
        const double xr = hx[2 * i], xi = hx[2 * i + 1];
        if (r->kode[i] == 0) {
          r->disp[2 * i] = r->bc[2 * i];
          r->disp[2 * i + 1] = r->bc[2 * i + 1];
          r->trac[2 * i] = xr * zge[0] - xi * zge[1];
          r->trac[2 * i + 1] = xr * zge[1] + xi * zge[0];
        } else {
          r->disp[2 * i] = xr;
          r->disp[2 * i + 1] = xi;
          r->trac[2 * i] = r->bc[2 * i];
          r->trac[2 * i + 1] = r->bc[2 * i + 1];
        }
      }
    }
    complete(r, st);
  }

  static bool same_problem(const Slot& s, const SrvRequest& r) {
    return s.cached && s.mesh == r.mesh && s.fr == r.fr && std::memcmp(s.mat, r.mat, sizeof s.mat) == 0 &&
           s.kode == r.kode;
  }

  void destroy_slot(Slot& s) {
    if (s.ctx) bem_ctx_destroy(s.ctx);
    if (s.done) cudaEventDestroy(s.done);
    if (s.h_x) pinned_free_.push_back({s.h_cap, s.h_x});  // kept: cudaFreeHost would stall the device
    used_bytes_ -= std::min(used_bytes_, s.bytes);
    s = Slot{};
  }

  // A pinned result buffer of at least `bytes`, from the ones earlier slots left.
  double* take_pinned(size_t bytes, size_t* cap) {
    size_t best = pinned_free_.size();
    for (size_t i = 0; i < pinned_free_.size(); ++i)
      if (pinned_free_[i].first >= bytes && (best == pinned_free_.size() || pinned_free_[i].first < pinned_free_[best].first))
        best = i;
    if (best < pinned_free_.size()) {
      auto b = pinned_free_[best];
      pinned_free_.erase(pinned_free_.begin() + (long)best);
      *cap = b.first;
      return b.second;
    }
    double* p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    *cap = bytes;
    return p;
  }

  // Frees idle slots, least recently used first, until `need` more bytes fit.
  bool make_room(size_t need) {
    while (used_bytes_ + need > budget_) {
      Slot* victim = nullptr;
      for (Slot& s : slots_)
        if (s.ctx && !s.busy && (!victim || s.last_use < victim->last_use)) victim = &s;
      if (!victim) return false;
      destroy_slot(*victim);
      ++n_evict_;
    }
    return true;
  }

  static uint64_t bits(double v) {
    uint64_t u;
    std::memcpy(&u, &v, sizeof u);
    return u;
  }

  // Key of a request's problem (mesh, material, boundary conditions, KODE):
  // requests with equal data get the same key.  A hash of the data picks the
  // bucket, one full comparison against a live request of the bucket decides,
  // so the queue scans compare keys only.  Buckets hold weak references: a
  // key outlives its requests only while one of them is alive.
  long long problem_key(const std::shared_ptr<SrvRequest>& r) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over 64- and 32-bit words
    auto mix = [&h](uint64_t w) { h = (h ^ w) * 1099511628211ull; };
    mix((uint64_t)r->mesh);
    for (double v : r->mat) mix(bits(v));
    for (double v : r->bc) mix(bits(v));
    for (int v : r->kode) mix((uint32_t)v);
    auto& bucket = pkeys_[h];
    for (auto it = bucket.begin(); it != bucket.end();) {
      auto q = it->lock();
      if (!q) {
        it = bucket.erase(it);
        continue;
      }
      if (q->mesh == r->mesh && std::memcmp(q->mat, r->mat, sizeof q->mat) == 0 && q->kode == r->kode &&
          q->bc == r->bc)
        return q->pkey;
      ++it;
    }
    bucket.push_back(r);
    // a long-running server sees ever new problems: drop the buckets whose
    // requests are all gone, now and then
    if ((++pkey_inserts_ & 1023u) == 0)
      for (auto b = pkeys_.begin(); b != pkeys_.end();) {
        auto& v = b->second;
        v.erase(std::remove_if(v.begin(), v.end(), [](const std::weak_ptr<SrvRequest>& w) { return w.expired(); }),
                v.end());
        b = v.empty() ? pkeys_.erase(b) : std::next(b);
      }
    return ++next_pkey_;
  }

  // Queued requests that can run in lockstep with r: same mesh, material,
  // boundary conditions and KODE, any omega (a frequency sweep).
  std::vector<std::shared_ptr<SrvRequest>> companions(const std::shared_ptr<SrvRequest>& r, int room) {
    std::vector<std::shared_ptr<SrvRequest>> out;
    for (const auto& q : queue_) {
      if ((int)out.size() + 1 >= room) break;
      if (q == r || q->started || q->pkey != r->pkey) continue;
      out.push_back(q);
    }
    return out;
  }

  // Problems in lockstep on one slot for an nn-unknown mesh: the panel
  // kernel's resident limit, at most kMaxBatch (a context of the server's
  // own answers the occupancy query and caches it per size).
  int lockstep_cap(int nn) {
    if (!probe_ && bem_ctx_create(device_, &probe_) != BEM_OK) {
      probe_ = nullptr;
      return 1;
    }
    std::lock_guard<std::mutex> g(probe_->mu);
    return std::max(1, std::min(kMaxBatch, lu_lockstep_capacity(probe_, nn, mixed_)));
  }

  // Problems started (the request, and those batched with it), 0 not yet
  // (waits for memory or a slot), -1 failed, kDefer: the request has more
  // lockstep companions queued than the in-flight limit lets start now
  // while other solves run, so it waits for a fuller batch (other requests
  // behind it may start meanwhile), for up to kDeferLimitMs.  `room`:
  // problems that may start.
  int try_start(const std::shared_ptr<SrvRequest>& r, int room) {
    const SrvMesh& m = meshes_[r->mesh];
    const int nn = 3 * m.nbe;
    Slot* slot = nullptr;
    bool rhs_only = false;
    for (Slot& s : slots_)
      if (s.ctx && !s.busy && same_problem(s, *r)) {
        slot = &s;
        rhs_only = true;
        break;
      }
    std::vector<std::shared_ptr<SrvRequest>> batch{r};
    if (!rhs_only) {
      // companions up to the lockstep limit, before any memory is reserved
      const int cap = lockstep_cap(nn);
      auto more = companions(r, cap);
      if ((int)more.size() + 1 > room) {
        const int target = std::min(cap, kMaxInflight);
        if (room < target && ms_between(r->t_submit, Clock::now()) < kDeferLimitMs) return kDefer;
        more.resize(room - 1);
      }
      batch.insert(batch.end(), more.begin(), more.end());
    }
    const size_t per = slot_footprint(nn, m.nbe, m.npg * m.npg, mixed_) +
                       (size_t)m.n * (m.npg * m.npg + 3) * sizeof(double4);
    if (!slot) {
      for (Slot& s : slots_)  // an idle slot of the same mesh: reuse its buffers
        if (s.ctx && !s.busy && s.mesh == r->mesh && (!slot || s.last_use < slot->last_use)) slot = &s;
    }
    if (slot && !rhs_only && (int)batch.size() > slot->cap_probs) {
      // a batch wider than the slot was admitted for: room for the difference, or one problem
      if (!make_room(per * (batch.size() - slot->cap_probs))) batch.resize(slot->cap_probs);
      else {
        used_bytes_ += per * (batch.size() - slot->cap_probs);
        peak_bytes_ = std::max(peak_bytes_, used_bytes_);
        slot->bytes += per * (batch.size() - slot->cap_probs);
        slot->cap_probs = (int)batch.size();
      }
    }
    if (!slot) {
      if (per > budget_) {
        complete(r, BEM_ERR_NOMEM);
        return -1;
      }
      while (batch.size() > 1 && per * batch.size() > budget_) batch.pop_back();
      if (!make_room(per * batch.size())) {
        batch.resize(1);
        if (!make_room(per)) return 0;
      }
      const size_t need = per * batch.size();
      Slot* fresh = nullptr;
      for (Slot& s : slots_)
        if (!s.ctx) {
          fresh = &s;
          break;
        }
      if (!fresh) {
        slots_.emplace_back();
        fresh = &slots_.back();
      }
      int st = bem_ctx_create(device_, &fresh->ctx);
      if (st == BEM_OK)
        st = bem_mesh_upload(fresh->ctx, m.n, m.nbe, m.np, m.npg, m.cone.data(), m.cx.data(), m.cy.data(),
                             m.cz.data(), m.cxm.data(), m.cym.data(), m.czm.data(), m.etas.data(), m.gi.data(),
                             m.ome.data());
      if (st == BEM_OK && cudaEventCreateWithFlags(&fresh->done, cudaEventDisableTiming) != cudaSuccess)
        st = BEM_ERR_CUDA;
      if (st != BEM_OK) {
        destroy_slot(*fresh);
        complete(r, st);
        return -1;
      }
      fresh->mesh = r->mesh;
      fresh->bytes = need;
      fresh->cap_probs = (int)batch.size();
      used_bytes_ += need;
      peak_bytes_ = std::max(peak_bytes_, used_bytes_);
      slot = fresh;
    }
    bem_ctx* ctx = slot->ctx;
    int st = BEM_OK;
    {
      double zge[2], zcs[2], zcp[2], c[4];
      material_consts(r->mat, zge, zcs, zcp);
      static_consts(r->mat[0], r->mat[1], c);
      st = bem_dyn_upload(ctx, r->bc.data(), r->kode.data());
      std::lock_guard<std::mutex> g(ctx->mu);
      cudaSetDevice(device_);
      if (batch.size() > 1)  // no more problems in lockstep than the panel kernel keeps resident
        batch.resize(std::min(batch.size(), (size_t)std::max(1, lu_lockstep_capacity(ctx, nn, mixed_))));
      const size_t hneed = 2 * (size_t)nn * sizeof(double) * batch.size();
      if (st == BEM_OK && slot->h_cap < hneed) {
        if (slot->h_x) pinned_free_.push_back({slot->h_cap, slot->h_x});
        slot->h_x = take_pinned(hneed, &slot->h_cap);
        if (!slot->h_x) st = BEM_ERR_NOMEM;
      }
      if (st == BEM_OK && !rhs_only && !(slot->have_static && slot->st_ge == r->mat[0] && slot->st_nu == r->mat[1])) {
        st = cudaMemsetAsync(ctx->d_status, 0, ST_COUNT * sizeof(int), ctx->stream) == cudaSuccess
                 ? launch_static(ctx, c, 1, nullptr)
                 : BEM_ERR_CUDA;
        if (st == BEM_OK) {
          ctx->have_hest = ctx->have_gest = true;
          slot->have_static = true;
          slot->st_ge = r->mat[0];
          slot->st_nu = r->mat[1];
        }
      }
      if (st == BEM_OK) {
        if (rhs_only) {
          st = slot_solve_rhs(ctx, mixed_, refine_);
        } else if (batch.size() == 1) {
          st = slot_solve_full(ctx, zge, zcs, zcp, c, r->fr, mixed_, refine_);
        } else {
          std::vector<double> fr;
          for (const auto& q : batch) fr.push_back(q->fr);
          st = slot_solve_batch(ctx, zge, zcs, zcp, c, fr.data(), (int)batch.size(), mixed_, refine_);
        }
      }
      for (size_t b = 0; b < batch.size() && st == BEM_OK; ++b) {
        const double2* x = batch.size() == 1 ? slot_solution(ctx, mixed_, rhs_only)
                                             : slot_batch_solution(ctx, mixed_, (int)b);
        if (cudaMemcpyAsync(slot->h_x + 2 * (size_t)nn * b, x, (size_t)nn * sizeof(double2), cudaMemcpyDeviceToHost,
                            ctx->stream) != cudaSuccess)
          st = BEM_ERR_CUDA;
      }
      if (st == BEM_OK && cudaEventRecord(slot->done, ctx->stream) != cudaSuccess) st = BEM_ERR_CUDA;
    }
    if (st != BEM_OK) {
      slot->cached = false;
      complete(r, st);
      return -1;
    }
    slot->busy = true;
    slot->cached = false;
    slot->reqs = batch;
    std::memcpy(slot->mat, r->mat, sizeof slot->mat);
    slot->fr = r->fr;
    slot->kode = r->kode;
    slot->last_use = ++tick_;
    const auto now = Clock::now();
    for (const auto& q : batch) {
      q->started = true;
      q->rhs_only = rhs_only;
      q->bytes = slot->bytes / batch.size();
      q->t_start = now;
    }
    return (int)batch.size();
  }

  int device_;
  bem_ctx* probe_ = nullptr;  // lockstep-limit queries (loop thread)
  size_t budget_;
  bool mixed_;
  int refine_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::thread worker_;
  bool stop_ = false;
  std::vector<SrvMesh> meshes_;
  std::deque<Slot> slots_;  // stable addresses
  std::vector<std::pair<size_t, double*>> pinned_free_;  // pinned buffers of destroyed slots
  std::deque<std::shared_ptr<SrvRequest>> queue_;
  std::unordered_map<long long, std::shared_ptr<SrvRequest>> reqs_;
  std::unordered_map<uint64_t, std::vector<std::weak_ptr<SrvRequest>>> pkeys_;  // problem_key's buckets
  long long next_id_ = 0, next_pkey_ = 0;
  unsigned pkey_inserts_ = 0;
  unsigned long long tick_ = 0;
  size_t used_bytes_ = 0, peak_bytes_ = 0;
  long long n_rhs_only_ = 0, n_evict_ = 0;
  int max_busy_ = 0;
  std::vector<double> lat_;
  Clock::time_point first_submit_, last_done_;
  bool have_first_ = false;
};

}  // namespace bem

struct bem_server {
  bem::Server* s;
};

using namespace bem;

int bem_server_create(int device, double budget_bytes, int form, int refine, bem_server** out) {
  if (!out || budget_bytes <= 0 || (form != BEM_FORM_PLAIN && form != BEM_FORM_MIXED) || refine < 0 ||
      refine > kMaxRefine)
    return BEM_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return BEM_ERR_CUDA;
  *out = new bem_server{new Server(device, budget_bytes, form, refine)};
  return BEM_OK;
}

int bem_server_destroy(bem_server* srv) {
  if (!srv) return BEM_OK;
  delete srv->s;
  delete srv;
  return BEM_OK;
}

int bem_server_add_mesh(bem_server* srv, int n, int nbe, int np, int npg, const int* cone, const double* cx,
                        const double* cy, const double* cz, const double* cxm, const double* cym, const double* czm,
                        const double* etas, const double* gi, const double* ome, int* mesh_id) {
  if (!srv || !mesh_id || n <= 0 || nbe <= 0 || nbe > n || np <= 0 || npg <= 0 || npg > kMaxNpg || !cone || !cx ||
      !cy || !cz || !cxm || !cym || !czm || !etas || !gi || !ome)
    return BEM_ERR_ARG;
  SrvMesh m;
  m.n = n;
  m.nbe = nbe;
  m.np = np;
  m.npg = npg;
  m.cone.assign(cone, cone + 4 * (size_t)n);
  m.cx.assign(cx, cx + np);
  m.cy.assign(cy, cy + np);
  m.cz.assign(cz, cz + np);
  m.cxm.assign(cxm, cxm + n);
  m.cym.assign(cym, cym + n);
  m.czm.assign(czm, czm + n);
  m.etas.assign(etas, etas + 3 * (size_t)n);
  m.gi.assign(gi, gi + npg);
  m.ome.assign(ome, ome + npg);
  *mesh_id = srv->s->add_mesh(std::move(m));
  return BEM_OK;
}

int bem_server_submit(bem_server* srv, int mesh_id, const double material[4], double fr, const double* bc,
                      const int* kode, long long* req_id) {
  if (!srv || !material || !bc || !kode || !req_id) return BEM_ERR_ARG;
  return srv->s->submit(mesh_id, material, fr, bc, kode, req_id);
}

int bem_server_wait(bem_server* srv, long long req_id, double timeout_s, double* disp, double* trac, double* info) {
  if (!srv) return BEM_ERR_ARG;
  return srv->s->wait(req_id, timeout_s, disp, trac, info);
}

int bem_server_stats(bem_server* srv, double* out) {
  if (!srv || !out) return BEM_ERR_ARG;
  srv->s->stats(out);
  return BEM_OK;
}

int bem_server_reset_stats(bem_server* srv) {
  if (!srv) return BEM_ERR_ARG;
  srv->s->reset_stats();
  return BEM_OK;
}
