// gd_serve.cu -- the request loop: docking jobs of different ligand sizes
// against resident pockets, admitted by an HBM budget into a running batch.
//
// Continuous batching at round granularity.  A round is one persistent Monte
// Carlo launch over every admitted job (each job runs min(round, steps to its
// next exchange, steps left) steps from its own step count), one exchange
// launch (each job with its own sweep index) and, for jobs admitted since the
// last round, one launch of initial energies before it.  Between rounds the
// scheduler thread retires finished jobs (results copied out, device memory
// and budget released) and admits queued ones while the budget, the replica
// cap and the job slots allow.  The host prepares round k+1 while round k runs;
// uploads go through a second stream with stream-ordered allocation, so an
// admission never synchronises the device.
//
// Every job keeps its own Philox key (its seed) and step counter, so its
// result does not depend on which other jobs shared its rounds.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "gd_internal.h"
#include "gd_pack.h"
#include "gdock.h"

using namespace gd;

namespace {

constexpr size_t kSmemLimitServe = 227 * 1024;
constexpr int kMaxServeSlots = 65535;  // exchange grid's y extent

using Clock = std::chrono::steady_clock;

struct ServeReq {
  long long ticket = 0;
  JobData jd;
  int pocket = 0, steps = 0, spx = 0, nrep = 0;
  size_t bytes = 0;
  ReplicaMC *out_rep = nullptr;
  double *out_stats = nullptr;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // admitted state
  int slot = -1;
  DevJobBuf buf;
  int step = 0;
  bool fresh = true;   // initial energies not evaluated yet
  bool done = false;   // final round enqueued, result not yet copied out
  int nstep_round = 0;
};

void stats_to_out8(const RepStats &x, double *o)
{
  const double n = (double)x.n_steps;
  o[0] = n;
  o[1] = (double)x.n_accept;
  o[2] = (double)x.n_exch_try;
  o[3] = (double)x.n_exch_acc;
  o[4] = n > 0 ? x.e_sum / n : 0.0;
  o[5] = n > 0 ? std::max(0.0, x.e_sum2 / n - o[4] * o[4]) : 0.0;
  o[6] = x.best_e;
  o[7] = (double)x.best_step;
}

}  // namespace

struct gd_server {
  int device = 0;
  gd_server_config_t cfg{};
  EnePara ep{};
  std::vector<DevPocket> pockets;
  cudaStream_t st = nullptr, up = nullptr;
  cudaEvent_t up_ev = nullptr;
  cudaEvent_t rev[2] = {nullptr, nullptr};
  cudaEvent_t t_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  TileConfig tc{8, 2, 8};
  int precision = GD_PREC_FP32;
  int grid = 0, Pmax = 0, Kst = 0, lig_slots = 0;
  size_t smem = 0;
  // adaptive latency mode (replica_warps = -G): the launch shapes of G, G/2, ...
  // 2 warps per replica, largest first, each with the replicas one wave holds
  struct Level {
    TileConfig tc{8, 2, 8};
    int grid = 0, Kst = 0;
    long long wave = 0;
  };
  Level lv[3];
  int nlv = 0;
  int max_items = 0;
  // device tables
  DevJob *d_jobs = nullptr;
  WorkItem *d_items = nullptr;
  int *d_queue = nullptr;
  int *d_err = nullptr;
  // pinned host mirrors (one per round parity) and result staging (per slot)
  DevJob *h_jobs[2] = {nullptr, nullptr};
  WorkItem *h_items[2] = {nullptr, nullptr};
  int *h_err = nullptr;
  unsigned char *h_stage = nullptr;
  size_t stage_per_slot = 0;
  // queues
  std::mutex mu;
  std::condition_variable cv_sub, cv_res, cv_idle;
  std::deque<std::unique_ptr<ServeReq>> pending;
  std::deque<gd_result_t> results;
  std::vector<long long> cancel;   // tickets of admitted requests to cancel at the next round boundary
  std::unordered_set<long long> live;  // tickets submitted and not yet reported
  long long next_ticket = 1;
  long long outstanding = 0;
  size_t used_bytes = 0;
  bool stop = false;
  int fatal = GD_OK;
  std::string fatal_msg;
  std::thread th;
  Clock::time_point t0;
  // scheduler-thread state
  std::vector<std::unique_ptr<ServeReq>> slots;  // [max_jobs]
  std::vector<int> free_slots;
  int active_reps = 0;
  // counters (under mu)
  gd_server_stats_t stats{};
};

namespace {

double now_s(const gd_server *s) { return std::chrono::duration<double>(Clock::now() - s->t0).count(); }

size_t estimate_bytes(const JobData &jd, const DevPocket &pk)
{
  const size_t L = jd.L, P = pk.Ppad, C = pk.nconf, nrep = jd.reps.size();
  const size_t lstride = (L + 3) & ~size_t(3);
  size_t b = C * kLigTypes * P * 4 + C * P * 4;                     // psp gather + masks
  b += jd.nlig * lstride * 16 + L * 8 + jd.nlig * 12;               // ligand
  b += std::max<size_t>(jd.K, 1) * 16 + L * jd.M * 16 + jd.M * 4;   // KDE, MCS
  b += jd.ntmp * 4 + sizeof(DevParams) + kLigTypes * kTabCols * 8;  // ladder, parameters
  b += nrep * (sizeof(ReplicaMC) + sizeof(int) + sizeof(RepStats));
  return b + 16 * 256;                                               // alignment
}

// Completes a request (error or result) and wakes pollers.  Caller holds mu.
void publish(gd_server *s, ServeReq &r, int status)
{
  gd_result_t res{};
  res.ticket = r.ticket;
  res.status = status;
  res.nrep = r.nrep;
  res.steps = r.step;
  res.t_submit = r.t_submit;
  res.t_admit = r.t_admit;
  res.t_done = now_s(s);
  s->results.push_back(res);
  s->live.erase(r.ticket);
  --s->outstanding;
  if (status == GD_OK) ++s->stats.completed;
  else ++s->stats.failed;
  s->cv_res.notify_all();
  if (s->outstanding == 0) s->cv_idle.notify_all();
}

void release(gd_server *s, ServeReq &r)
{
  s->used_bytes -= r.bytes;
  if (r.slot >= 0) s->free_slots.push_back(r.slot);
}

// Fails every queued and admitted request (fatal device error or shutdown).
void fail_all(gd_server *s, int status)
{
  std::lock_guard<std::mutex> lk(s->mu);
  while (!s->pending.empty()) {
    publish(s, *s->pending.front(), status);
    s->pending.pop_front();
  }
  for (auto &p : s->slots)
    if (p) {
      if (p->buf.arena) free_job(p->buf);  // the caller synchronised the streams
      release(s, *p);
      publish(s, *p, status);
      p.reset();
    }
}

int set_fatal(gd_server *s, int rc)
{
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->fatal == GD_OK) {
    s->fatal = rc;
    s->fatal_msg = gd_last_error();
  }
  return rc;
}

// Copies finished requests' staged results out and publishes them.
void complete(gd_server *s, std::vector<ServeReq *> &done)
{
  std::lock_guard<std::mutex> lk(s->mu);
  for (ServeReq *r : done) {
    const unsigned char *stg = s->h_stage + (size_t)r->slot * s->stage_per_slot;
    const ReplicaMC *rep = reinterpret_cast<const ReplicaMC *>(stg);
    const RepStats *rs = reinterpret_cast<const RepStats *>(stg + sizeof(ReplicaMC) * r->nrep);
    if (r->out_rep) std::memcpy(r->out_rep, rep, sizeof(ReplicaMC) * r->nrep);
    if (r->out_stats)
      for (int i = 0; i < r->nrep; ++i) stats_to_out8(rs[i], r->out_stats + 8 * (size_t)i);
    const int slot = r->slot;
    release(s, *r);
    publish(s, *r, GD_OK);
    s->slots[slot].reset();
  }
  done.clear();
}

// Items of one launch: runs of consecutive replicas with the same protein
// conformation, at most warps_per_cta long, heaviest job first.
void append_items(const TileConfig &tc, const ServeReq &r, std::vector<WorkItem> &out)
{
  const int R = tc.warps_per_cta / tc.group;  // replicas per CTA
  const std::vector<ReplicaMC> &reps = r.jd.reps;
  int i = 0;
  while (i < r.nrep) {
    int k = 1;
    while (i + k < r.nrep && k < R && reps[i + k].idx_prt == reps[i].idx_prt) ++k;
    out.push_back(WorkItem{r.slot, reps[i].idx_prt, i, k});
    i += k;
  }
}

int enqueue_round(gd_server *s, long long k, std::vector<ServeReq *> &finishing, bool &enqueued)
{
  enqueued = false;
  const int b = (int)(k & 1);
  std::vector<ServeReq *> act;
  for (auto &p : s->slots)
    if (p && !p->done) act.push_back(p.get());
  if (act.empty()) return GD_OK;
  const int R = s->cfg.steps_per_round;
  int nmax = 0, nslot = 0, max_pairs = 0;
  bool any_fresh = false;
  long long nrep_act = 0;
  for (ServeReq *r : act) {
    int n = std::min(R, r->steps - r->step);
    if (r->spx > 0) n = std::min(n, r->spx - r->step % r->spx);
    r->nstep_round = n;
    nmax = std::max(nmax, n);
    nslot = std::max(nslot, r->slot + 1);
    any_fresh |= r->fresh;
    nrep_act += r->nrep;
  }
  // adaptive latency mode: the most warps per replica whose one wave holds the
  // round's replicas; one warp per replica when none does
  int li = -1;
  for (int i = 0; i < s->nlv && li < 0; ++i)
    if (nrep_act <= s->lv[i].wave) li = i;
  const bool lat = li >= 0;
  const TileConfig &tc = lat ? s->lv[li].tc : s->tc;
  const int grid = lat ? s->lv[li].grid : s->grid;
  // job table of this round
  DevJob *hj = s->h_jobs[b];
  for (int i = 0; i < nslot; ++i) hj[i] = DevJob{};
  for (int i = 0; i < nslot; ++i) hj[i].xsweep = -1;
  for (ServeReq *r : act) {
    DevJob J = r->buf.dj;
    J.step0 = r->step;
    J.nsteps = std::max(r->nstep_round, 1);
    const int after = r->step + r->nstep_round;
    J.xsweep = (r->spx > 0 && r->nstep_round > 0 && after % r->spx == 0) ? after / r->spx - 1 : -1;
    if (J.xsweep >= 0 && J.ntmp >= 2) max_pairs = std::max(max_pairs, J.nprt * J.nlig * (J.ntmp / 2));
    hj[r->slot] = J;
  }
  // items: the round's chunk first, then the initial evaluation of new jobs
  std::vector<ServeReq *> ord(act);
  std::stable_sort(ord.begin(), ord.end(), [](const ServeReq *a, const ServeReq *c) {
    return (double)a->jd.L * a->buf.dj.npoint_pad > (double)c->jd.L * c->buf.dj.npoint_pad;
  });
  std::vector<WorkItem> items, init;
  for (ServeReq *r : ord) {
    if (r->nstep_round > 0) append_items(tc, *r, items);
    if (r->fresh) append_items(tc, *r, init);
  }
  const int n_chunk = (int)items.size(), n_init = (int)init.size();
  if (n_chunk + n_init > s->max_items) return fail(GD_E_CAPACITY, "round of %d work items", n_chunk + n_init);
  std::memcpy(s->h_items[b], items.data(), sizeof(WorkItem) * n_chunk);
  std::memcpy(s->h_items[b] + n_chunk, init.data(), sizeof(WorkItem) * n_init);

  GD_CUDA(cudaMemcpyAsync(s->d_jobs, hj, sizeof(DevJob) * nslot, cudaMemcpyHostToDevice, s->st));
  GD_CUDA(cudaMemcpyAsync(s->d_items, s->h_items[b], sizeof(WorkItem) * (n_chunk + n_init), cudaMemcpyHostToDevice,
                          s->st));
  KArgs a{};
  a.jobs = s->d_jobs;
  a.queue = s->d_queue;
  a.err = s->d_err;
  a.P = tc.stage ? s->Pmax : 0;
  a.Kst = lat ? s->lv[li].Kst : s->Kst;
  a.lig_slots = s->lig_slots;
  a.group = (uint16_t)tc.group;
  int launches = 0;
  GD_CUDA(cudaEventRecord(s->t_ev[b][0], s->st));
  if (any_fresh) {
    a.items = s->d_items + n_chunk;
    a.n_items = n_init;
    a.s_begin = 0;
    a.nsteps = 1;
    a.flags = kMcInitial | kMcStoreAccept;
    GD_CUDA(cudaMemsetAsync(s->d_queue, 0, sizeof(int), s->st));
    GD_CUDA(launch_kernel(0, s->precision, tc, a, std::max(1, std::min(grid, n_init)), s->st));
    ++launches;
  }
  if (n_chunk > 0) {
    a.items = s->d_items;
    a.n_items = n_chunk;
    a.s_begin = 0;
    a.nsteps = nmax;
    a.flags = kMcStoreAccept;
    GD_CUDA(cudaMemsetAsync(s->d_queue, 0, sizeof(int), s->st));
    GD_CUDA(launch_kernel(0, s->precision, tc, a, std::max(1, std::min(grid, n_chunk)), s->st));
    ++launches;
  }
  if (max_pairs > 0) {
    GD_CUDA(launch_exchange_jobs(s->d_jobs, nslot, max_pairs, s->st));
    ++launches;
  }
  GD_CUDA(cudaEventRecord(s->t_ev[b][1], s->st));

  double evals = 0;
  for (ServeReq *r : act) {
    evals += (double)r->nrep * (r->nstep_round + (r->fresh ? 1 : 0));
    r->step += r->nstep_round;
    r->fresh = false;
    if (r->step >= r->steps) {
      unsigned char *stg = s->h_stage + (size_t)r->slot * s->stage_per_slot;
      GD_CUDA(cudaMemcpyAsync(stg, r->buf.dj.rep, sizeof(ReplicaMC) * r->nrep, cudaMemcpyDeviceToHost, s->st));
      GD_CUDA(cudaMemcpyAsync(stg + sizeof(ReplicaMC) * r->nrep, r->buf.dj.stats, sizeof(RepStats) * r->nrep,
                              cudaMemcpyDeviceToHost, s->st));
      free_job_async(r->buf, s->st);
      r->done = true;
      finishing.push_back(r);
    }
  }
  GD_CUDA(cudaMemcpyAsync(s->h_err + b, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  GD_CUDA(cudaEventRecord(s->rev[b], s->st));
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.rounds += 1;
    s->stats.latency_rounds += lat ? 1 : 0;
    s->stats.launches += launches;
    s->stats.pose_evals += evals;
    for (ServeReq *r : finishing) s->active_reps -= r->nrep;
  }
  enqueued = true;
  return GD_OK;
}

// Takes queued requests while the budget, the replica cap and the slots
// allow, in submission order.  A request alone always fits both (checked at
// submission).  Memory of a finished request counts against the budget until
// its result has been copied out; its replicas leave the cap when its last
// round is enqueued.
int admit(gd_server *s)
{
  std::vector<std::unique_ptr<ServeReq>> take;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    while (!s->pending.empty()) {
      ServeReq &r = *s->pending.front();
      if (s->free_slots.empty()) break;
      if (s->active_reps + r.nrep > s->cfg.max_active_replicas) break;
      if (s->used_bytes + r.bytes > s->cfg.hbm_budget_bytes) break;
      s->used_bytes += r.bytes;
      s->stats.peak_bytes = std::max(s->stats.peak_bytes, (unsigned long long)s->used_bytes);
      s->active_reps += r.nrep;
      r.slot = s->free_slots.back();
      s->free_slots.pop_back();
      take.push_back(std::move(s->pending.front()));
      s->pending.pop_front();
    }
  }
  if (take.empty()) return GD_OK;
  for (auto &p : take) {
    ServeReq &r = *p;
    const int rc = pack_job_async(r.jd, s->pockets[r.pocket], s->ep, s->up, r.buf);
    r.t_admit = now_s(s);
    if (rc != GD_OK) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->active_reps -= r.nrep;
      release(s, r);
      publish(s, r, rc);
      continue;
    }
    r.jd.lxyz.clear();  // host copies no longer needed (replica layout is kept for the items)
    r.jd.psp.clear();
    r.jd.mxyz.clear();
    s->slots[r.slot] = std::move(p);
  }
  GD_CUDA(cudaEventRecord(s->up_ev, s->up));
  GD_CUDA(cudaStreamWaitEvent(s->st, s->up_ev, 0));
  return GD_OK;
}

// Retires the admitted requests whose cancellation was asked for: their
// memory is freed stream-ordered after the rounds already enqueued (which
// still name them), and they are reported as GD_E_CANCELLED.  A request whose
// final round is already enqueued finishes normally.
void retire_cancelled(gd_server *s)
{
  std::vector<long long> ask;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->cancel.empty()) return;
    ask.swap(s->cancel);
  }
  for (long long t : ask)
    for (auto &p : s->slots)
      if (p && p->ticket == t && !p->done) {
        free_job_async(p->buf, s->st);
        std::lock_guard<std::mutex> lk(s->mu);
        s->active_reps -= p->nrep;
        release(s, *p);
        publish(s, *p, GD_E_CANCELLED);
        p.reset();
        break;
      }
}

void serve_loop(gd_server *s)
{
  if (cudaSetDevice(s->device) != cudaSuccess) {
    set_fatal(s, fail(GD_E_CUDA, "cudaSetDevice(%d) in the server thread", s->device));
    fail_all(s, GD_E_CUDA);
    return;
  }
  long long k = 0;
  std::vector<ServeReq *> fin_prev, fin_cur;
  bool prev = false;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      auto nothing = [&] { return s->pending.empty() && s->active_reps == 0 && s->cancel.empty(); };
      while (!s->stop && nothing() && !prev) s->cv_sub.wait_for(lk, std::chrono::milliseconds(50));
      if (s->stop) break;
    }
    retire_cancelled(s);
    int rc = admit(s);
    bool enq = false;
    if (rc == GD_OK) rc = enqueue_round(s, k, fin_cur, enq);
    if (rc == GD_OK && prev) {
      const int pb = (int)((k - 1) & 1);
      const cudaError_t ce = cudaEventSynchronize(s->rev[pb]);
      if (ce != cudaSuccess) rc = fail(GD_E_CUDA, "round %lld: %s", k - 1, cudaGetErrorString(ce));
      else if (s->h_err[pb] & kErrTimeout) rc = fail(GD_E_TIMEOUT, "a bounded wait for a shared-memory bulk copy gave up");
      if (rc == GD_OK) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, s->t_ev[pb][0], s->t_ev[pb][1]) == cudaSuccess) {
          std::lock_guard<std::mutex> lk(s->mu);
          s->stats.device_ms += ms;
        }
        complete(s, fin_prev);
      }
    }
    if (rc != GD_OK) {
      set_fatal(s, rc);
      cudaStreamSynchronize(s->st);
      fail_all(s, rc);
      return;
    }
    fin_prev.swap(fin_cur);
    fin_cur.clear();
    prev = enq;
    if (enq) ++k;
  }
  // shutdown: let the last round land, then cancel what is left
  cudaStreamSynchronize(s->st);
  cudaStreamSynchronize(s->up);
  fin_prev.clear();
  fail_all(s, GD_E_CANCELLED);
}

// Launch shape of tile tc's group: warps per CTA and pocket staging from the
// resident replica-warps per SM; sets tc, grid, Kst, smem and the CTAs per SM.
int choose_shape(gd_server *s, TileConfig &tc_out, int &grid, int &Kst, size_t &smem_out, int &occ_out)
{
  int nsm = 0;
  GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->device));
  const int G = tc_out.group;
  const int w0 = s->cfg.warps, wlo = w0 > 0 ? w0 : std::max(2, G), whi = w0 > 0 ? w0 : kMaxCtaThreads / 32;
  int best_w = 0, best_res = 0, best_occ = 0, best_kst = 0, best_stage = 1;
  size_t best_smem = 0;
  // resident replica-warps per SM decide; the pocket is staged in shared
  // memory unless reading it through L1 lets more replicas be resident
  for (int stage = 1; stage >= 0; --stage)
  for (int w = wlo; w <= whi; ++w) {
    if (w % G) continue;
    TileConfig tc = tc_out;
    tc.warps_per_cta = w;
    tc.stage = stage;
    const int P = stage ? s->Pmax : 0;
    int kst = s->cfg.kde_stage;
    size_t smem = kernel_smem_bytes(P, kst, s->lig_slots, w, s->precision, G);
    if (smem > kSmemLimitServe) {
      kst = 0;
      smem = kernel_smem_bytes(P, kst, s->lig_slots, w, s->precision, G);
    }
    if (smem > kSmemLimitServe) continue;
    const int occ = kernel_occupancy(0, s->precision, tc, smem);
    if (occ < 1) continue;
    const int resident = std::min(occ * w, 32);
    if (resident > best_res || (resident == best_res && stage == best_stage && kst > best_kst)) {
      best_res = resident;
      best_w = w;
      best_occ = occ;
      best_smem = smem;
      best_kst = kst;
      best_stage = stage;
    }
  }
  if (best_w == 0) return fail(GD_E_CAPACITY, "no launch shape fits shared memory");
  tc_out.warps_per_cta = best_w;
  tc_out.stage = best_stage;
  Kst = best_kst;
  smem_out = best_smem;
  grid = best_occ * nsm;
  occ_out = best_occ;
  return GD_OK;
}

int server_configure(gd_server *s)
{
  int occ = 0;
  GD_TRY(choose_shape(s, s->tc, s->grid, s->Kst, s->smem, occ));
  // four waves of resident replica-warps per round: more balanced rounds (items
  // of uneven jobs) than two, with the same latency below saturation
  if (s->cfg.max_active_replicas <= 0)
    s->cfg.max_active_replicas = 4 * s->grid * (s->tc.warps_per_cta / s->tc.group);
  for (int i = 0; i < s->nlv; ++i) {
    gd_server::Level &l = s->lv[i];
    size_t smem_l = 0;
    int occ_l = 0;
    GD_TRY(choose_shape(s, l.tc, l.grid, l.Kst, smem_l, occ_l));
    l.wave = (long long)l.grid * (l.tc.warps_per_cta / l.tc.group);
  }
  return GD_OK;
}

void server_free(gd_server *s)
{
  for (auto &p : s->pockets) free_pocket(p);
  for (auto &p : s->slots)
    if (p && p->buf.arena) free_job(p->buf);
  if (s->d_jobs) cudaFree(s->d_jobs);
  if (s->d_items) cudaFree(s->d_items);
  if (s->d_queue) cudaFree(s->d_queue);
  if (s->d_err) cudaFree(s->d_err);
  for (int b = 0; b < 2; ++b) {
    if (s->h_jobs[b]) cudaFreeHost(s->h_jobs[b]);
    if (s->h_items[b]) cudaFreeHost(s->h_items[b]);
    if (s->rev[b]) cudaEventDestroy(s->rev[b]);
    for (int i = 0; i < 2; ++i)
      if (s->t_ev[b][i]) cudaEventDestroy(s->t_ev[b][i]);
  }
  if (s->h_err) cudaFreeHost(s->h_err);
  if (s->h_stage) cudaFreeHost(s->h_stage);
  if (s->up_ev) cudaEventDestroy(s->up_ev);
  if (s->st) cudaStreamDestroy(s->st);
  if (s->up) cudaStreamDestroy(s->up);
  delete s;
}

int server_create(const gd_pocket_desc_t *pockets, int npocket, const EnePara *ep, const gd_server_config_t *cfg,
                  gd_server *s)
{
  GD_CUDA(cudaSetDevice(s->device));
  s->ep = *ep;
  for (int i = 0; i < npocket; ++i) {
    PocketData pd;
    GD_TRY(pocket_from_desc(pockets[i], pd));
    pd.hdb_types = hdb_point_types(s->ep);
    DevPocket dp;
    GD_TRY(pack_pocket(pd, dp));
    s->pockets.push_back(dp);
    s->Pmax = std::max(s->Pmax, dp.Ppad);
  }
  s->lig_slots = (s->cfg.max_atoms + 3) & ~3;
  const long long o_kpl = gd_get_option("kpl"), o_ab = gd_get_option("ab");
  s->precision = (int)gd_get_option("precision");
  s->tc = TileConfig{8, (int)o_kpl, (int)o_ab};
  const int rw = s->cfg.replica_warps;
  const int adapt = rw < 0 ? -rw : 0;
  s->tc.group = rw > 0 ? rw : 1;
  if (s->tc.group != 1 && s->tc.group != 2 && s->tc.group != 4 && s->tc.group != 8)
    return fail(GD_E_INVALID, "replica_warps = %d (1, 2, 4 or 8; -2, -4 or -8: adaptive)", rw);
  if (adapt && adapt != 2 && adapt != 4 && adapt != 8)
    return fail(GD_E_INVALID, "replica_warps = %d (1, 2, 4 or 8; -2, -4 or -8: adaptive)", rw);
  default_pair_tile(s->tc.group, s->tc.kpl, s->tc.ab);
  if (s->precision == GD_PREC_FP64) s->tc.kpl = 1, s->tc.ab = 8, s->tc.group = 1;
  if (s->tc.kpl % 2) s->tc.group = 1;  // the split form exists for the FP32 atom-pair loop
  s->nlv = 0;
  for (int g = adapt; g >= 2 && s->precision != GD_PREC_FP64; g /= 2) {
    TileConfig t{8, (int)o_kpl, (int)o_ab};
    t.group = g;
    default_pair_tile(g, t.kpl, t.ab);
    if (t.kpl % 2) break;  // the split form exists for the FP32 atom-pair loop
    s->lv[s->nlv++].tc = t;
  }
  GD_TRY(server_configure(s));
  s->max_items = s->cfg.max_active_replicas * 2 + s->cfg.max_replicas_per_job;
  GD_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  GD_CUDA(cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking));
  GD_CUDA(cudaEventCreateWithFlags(&s->up_ev, cudaEventDisableTiming));
  for (int b = 0; b < 2; ++b) {
    GD_CUDA(cudaEventCreateWithFlags(&s->rev[b], cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) GD_CUDA(cudaEventCreate(&s->t_ev[b][i]));
    GD_CUDA(cudaHostAlloc(&s->h_jobs[b], sizeof(DevJob) * s->cfg.max_jobs, cudaHostAllocDefault));
    GD_CUDA(cudaHostAlloc(&s->h_items[b], sizeof(WorkItem) * s->max_items, cudaHostAllocDefault));
  }
  GD_CUDA(cudaHostAlloc(&s->h_err, sizeof(int) * 2, cudaHostAllocDefault));
  s->h_err[0] = s->h_err[1] = 0;
  s->stage_per_slot = ((sizeof(ReplicaMC) + sizeof(RepStats)) * (size_t)s->cfg.max_replicas_per_job + 255) & ~size_t(255);
  GD_CUDA(cudaHostAlloc(&s->h_stage, s->stage_per_slot * s->cfg.max_jobs, cudaHostAllocDefault));
  GD_CUDA(cudaMalloc(&s->d_jobs, sizeof(DevJob) * s->cfg.max_jobs));
  GD_CUDA(cudaMalloc(&s->d_items, sizeof(WorkItem) * s->max_items));
  GD_CUDA(cudaMalloc(&s->d_queue, sizeof(int)));
  GD_CUDA(cudaMalloc(&s->d_err, sizeof(int)));
  GD_CUDA(cudaMemset(s->d_err, 0, sizeof(int)));
  // keep freed job memory in the stream-ordered pool instead of returning it each round
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
    uint64_t keep = std::min<uint64_t>(s->cfg.hbm_budget_bytes, 8ull << 30);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  s->slots.resize(s->cfg.max_jobs);
  for (int i = s->cfg.max_jobs - 1; i >= 0; --i) s->free_slots.push_back(i);
  GD_CUDA(cudaDeviceSynchronize());
  return GD_OK;
}

}  // namespace

extern "C" {

void gd_server_config_default(gd_server_config_t *cfg)
{
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->hbm_budget_bytes = 100ull * 1000 * 1000 * 1000;
  cfg->max_active_replicas = 0;
  cfg->max_jobs = 256;
  cfg->max_replicas_per_job = 1024;
  cfg->max_atoms = kMaxAtoms;
  cfg->steps_per_round = 50;
  cfg->kde_stage = 0;  // FP32 reads the KDE points through L1
  cfg->warps = 0;
  cfg->replica_warps = 1;
  cfg->device = 0;
}

int gd_server_create(const gd_pocket_desc_t *pockets, int npocket, const EnePara *enepara,
                     const gd_server_config_t *cfg, gd_server_t **out)
{
  if (!out) return fail(GD_E_INVALID, "null output handle");
  *out = nullptr;
  if (!pockets || npocket < 1 || !enepara) return fail(GD_E_INVALID, "server: %d pockets", npocket);
  gd_server_config_t c;
  gd_server_config_default(&c);
  if (cfg) c = *cfg;
  if (c.hbm_budget_bytes == 0 || c.max_jobs < 1 || c.max_jobs > kMaxServeSlots || c.max_replicas_per_job < 1 ||
      c.max_atoms < 1 || c.max_atoms > kMaxAtoms || c.steps_per_round < 1 || c.kde_stage < 0 || c.warps < 0 ||
      c.warps * 32 > kMaxCtaThreads || c.max_active_replicas < 0)
    return fail(GD_E_INVALID, "server configuration out of range");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return fail(GD_E_NODEVICE, "no CUDA device");
  if (c.device < 0 || c.device >= count) return fail(GD_E_INVALID, "device %d of %d", c.device, count);
  gd_server *s = new gd_server();
  s->cfg = c;
  s->device = c.device;
  s->t0 = Clock::now();
  const int rc = server_create(pockets, npocket, enepara, &c, s);
  if (rc != GD_OK) {
    server_free(s);
    return rc;
  }
  s->th = std::thread(serve_loop, s);
  *out = s;
  return GD_OK;
}

int gd_server_submit(gd_server_t *s, const gd_request_t *req, long long *ticket)
{
  if (!s || !req || !req->job) return fail(GD_E_INVALID, "null server or request");
  const gd_job_desc_t &d = *req->job;
  if (d.pocket < 0 || d.pocket >= (int)s->pockets.size())
    return fail(GD_E_INVALID, "request: pocket %d of %zu", d.pocket, s->pockets.size());
  if (req->steps < 0 || req->steps_per_exchange < 0)
    return fail(GD_E_INVALID, "request: steps = %d, steps_per_exchange = %d", req->steps, req->steps_per_exchange);
  if (d.natom > s->cfg.max_atoms) return fail(GD_E_CAPACITY, "request: %d atoms (server limit %d)", d.natom, s->cfg.max_atoms);
  auto r = std::make_unique<ServeReq>();
  GD_TRY(job_from_desc(d, s->pockets[d.pocket].nconf, r->jd));
  r->nrep = (int)r->jd.reps.size();
  if (r->nrep > s->cfg.max_replicas_per_job)
    return fail(GD_E_CAPACITY, "request: %d replicas (server limit %d)", r->nrep, s->cfg.max_replicas_per_job);
  if (r->nrep > s->cfg.max_active_replicas)
    return fail(GD_E_CAPACITY, "request: %d replicas above the per-round cap %d", r->nrep, s->cfg.max_active_replicas);
  r->pocket = d.pocket;
  r->steps = req->steps;
  r->spx = req->steps_per_exchange;
  r->out_rep = req->replicas_out;
  r->out_stats = req->stats_out;
  r->bytes = estimate_bytes(r->jd, s->pockets[d.pocket]);
  if (r->bytes > s->cfg.hbm_budget_bytes)
    return fail(GD_E_CAPACITY, "request needs %zu B, above the HBM budget", r->bytes);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->fatal != GD_OK) return fail(s->fatal, "server stopped: %s", s->fatal_msg.c_str());
  if (s->stop) return fail(GD_E_STATE, "server is shutting down");
  r->ticket = s->next_ticket++;
  s->live.insert(r->ticket);
  r->t_submit = now_s(s);
  if (ticket) *ticket = r->ticket;
  ++s->outstanding;
  ++s->stats.submitted;
  s->pending.push_back(std::move(r));
  s->cv_sub.notify_all();
  return GD_OK;
}

int gd_server_cancel(gd_server_t *s, long long ticket)
{
  if (!s) return fail(GD_E_INVALID, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
    if ((*it)->ticket == ticket) {
      publish(s, **it, GD_E_CANCELLED);
      s->pending.erase(it);
      return GD_OK;
    }
  if (ticket < 1 || ticket >= s->next_ticket) return fail(GD_E_INVALID, "cancel: unknown ticket %lld", ticket);
  if (!s->live.count(ticket)) return fail(GD_E_STATE, "cancel: request %lld already finished", ticket);
  s->cancel.push_back(ticket);
  s->cv_sub.notify_all();
  return GD_OK;
}

int gd_server_poll(gd_server_t *s, gd_result_t *out, int max, int timeout_ms)
{
  if (!s || !out || max < 1) return fail(GD_E_INVALID, "poll: null argument or max = %d", max);
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->results.empty() && timeout_ms != 0) {
    auto ready = [&] { return !s->results.empty() || s->outstanding == 0; };
    if (timeout_ms < 0) s->cv_res.wait(lk, ready);
    else s->cv_res.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
  }
  int n = 0;
  while (n < max && !s->results.empty()) {
    out[n++] = s->results.front();
    s->results.pop_front();
  }
  return n;
}

int gd_server_drain(gd_server_t *s, int timeout_ms)
{
  if (!s) return fail(GD_E_INVALID, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto idle = [&] { return s->outstanding == 0; };
  if (timeout_ms < 0) s->cv_idle.wait(lk, idle);
  else if (!s->cv_idle.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle))
    return fail(GD_E_TIMEOUT, "drain: %lld requests outstanding after %d ms", s->outstanding, timeout_ms);
  if (s->fatal != GD_OK) return fail(s->fatal, "server stopped: %s", s->fatal_msg.c_str());
  return GD_OK;
}

int gd_server_get_stats(gd_server_t *s, gd_server_stats_t *out)
{
  if (!s || !out) return fail(GD_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->now = now_s(s);
  out->queued = (long long)s->pending.size();
  out->outstanding = s->outstanding;
  out->used_bytes = s->used_bytes;
  out->warps_per_cta = s->tc.warps_per_cta;
  out->pocket_staged = s->tc.stage;
  out->grid = s->grid;
  out->max_active_replicas = s->cfg.max_active_replicas;
  return GD_OK;
}

int gd_server_destroy(gd_server_t *s)
{
  if (!s) return GD_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_sub.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  cudaSetDevice(s->device);
  server_free(s);
  return GD_OK;
}

}  // extern "C"
