// gd_api.cu -- the C ABI of libgdock.so: resident ensembles, the drop-in
// Dock family, and pose evaluation.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "gd_pack.h"

using namespace gd;

namespace {

struct Options {
  int kernel = GD_KERNEL_BATCHED;
  int precision = GD_PREC_FP32_KAHAN;  // FP32 pair terms, compensated reductions
  int warps = 0;  // 0: choose from occupancy
  int kpl = 0;    // pair-tile shape, 0: default_pair_tile
  int ab = 0;
  int graph = 1;  // replay whole exchange intervals from a captured graph
  int stage = -1; // protein conformation in shared memory: 1 staged, 0 through L1, -1 chosen
  int dock_cache = 1;  // Dock keeps its device state per GPU between calls
  int dock_device_pack = 1;  // Dock refills that state on the GPU from the Complex CopyH2D put there
  int dock_record_direct = 1;  // Dock's kernels write Records straight into a GPU-mapped host array
  int replica_warps = 1;     // warps per replica (1, 2, 4, 8): latency mode of the batched FP32 kernel
  int device_base = 0;        // the drop-in API's GPU g is CUDA device device_base + g
  long long wait_limit = 0;   // microseconds of a bounded shared-memory wait (0: one second)
  int stall_test = 0;         // test hook: staging barriers that never complete (bounded waits run out)
};
Options g_opt;
int g_ngpu = -1;
std::mutex g_mu;

int ngpu()
{
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_ngpu < 0) {
    const char *e = std::getenv("GDOCK_NGPU");
    g_ngpu = e ? std::max(1, std::atoi(e)) : 1;
  }
  return g_ngpu;
}

Options opts()
{
  std::lock_guard<std::mutex> lk(g_mu);
  return g_opt;
}

// Field by field: Options has padding, whose bytes a copy need not keep.
bool same_options(const Options &a, const Options &b)
{
  return a.kernel == b.kernel && a.precision == b.precision && a.warps == b.warps && a.kpl == b.kpl &&
         a.ab == b.ab && a.graph == b.graph && a.stage == b.stage && a.dock_cache == b.dock_cache &&
         a.dock_device_pack == b.dock_device_pack && a.replica_warps == b.replica_warps &&
         a.device_base == b.device_base && a.wait_limit == b.wait_limit && a.stall_test == b.stall_test;
}

constexpr size_t kSmemLimit = 227 * 1024;

}  // namespace

struct gd_ensemble;

struct gd_rng {
  uint64_t seed = 0;
  uint64_t calls = 0;
  int seeded = 0;
  uint64_t dock_calls = 0;   // Dock calls on this handle's GPU
  uint64_t dock_reused = 0;  // of them, refills of the kept device state
  // Dock's resident state on this handle's GPU, kept between calls and refilled
  // in place when the next Complex has the same shapes
  gd_ensemble *dock = nullptr;
  std::vector<unsigned char> dock_prt;  // protein bytes the cached pocket was packed from
  Options dock_opt;                     // options the cached ensemble was configured with
};

struct gd_ensemble {
  int device = 0;
  cudaStream_t st = nullptr;
  std::vector<DevPocket> pockets;
  std::vector<DevJobBuf> jobs;
  std::vector<std::vector<int>> rep_prt;  // per job, per replica: protein conformation
  DevJob *d_jobs = nullptr;
  WorkItem *d_items = nullptr;
  int n_items = 0;
  std::vector<WorkItem> h_items;   // host copy of d_items (the autotuner samples it)
  int *d_queue = nullptr;
  int *d_err = nullptr;
  int kernel = GD_KERNEL_BATCHED;
  int precision = GD_PREC_FP32;
  TileConfig tc{8, 1, 8};
  int grid = 0;
  size_t smem = 0;
  int Pmax = 0, Kmax = 0, Kst = 0, lig_slots = 0;
  int step = 0;
  // replica exchange over all jobs: pair-count prefix sums per parity
  int *d_xoff = nullptr;
  int xtot = 0;
  // device copy of the step counter and the captured exchange interval
  int *d_step = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int g_chunk = 0;
  bool use_graph = true;
  // timing of the Monte Carlo launches
  std::vector<cudaEvent_t> ev;
  int ev_used = 0;
  uint32_t wait_limit = 0, stall_bytes = 0;  // bounded-wait limit and the test hook (options)
  int launches = 0;      // Monte Carlo kernel launches (or graph replays of one)
  int all_launches = 0;  // every kernel of this library launched on the stream
};

namespace {

int set_device(int d) { GD_CUDA(cudaSetDevice(d)); return GD_OK; }

// CUDA device of the drop-in API's GPU g.
int dev_of(int g) { return opts().device_base + g; }

// Work items: runs of consecutive replicas of one job with the same protein
// conformation, at most `warps` long; heaviest (L x P) first.
int build_items(gd_ensemble *e)
{
  std::vector<WorkItem> items;
  std::vector<double> cost;
  const int R = e->tc.warps_per_cta / std::max(1, e->tc.group);  // replicas per CTA
  for (int j = 0; j < (int)e->jobs.size(); ++j) {
    const std::vector<int> &pr = e->rep_prt[j];
    const double c = (double)e->jobs[j].dj.natom * e->jobs[j].dj.npoint_pad;
    int r = 0;
    const int n = (int)pr.size();
    while (r < n) {
      int k = 1;
      while (r + k < n && k < R && pr[r + k] == pr[r]) ++k;
      items.push_back(WorkItem{j, pr[r], r, k});
      cost.push_back(c);
      r += k;
    }
  }
  std::vector<int> ord(items.size());
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<WorkItem> sorted(items.size());
  for (size_t i = 0; i < ord.size(); ++i) sorted[i] = items[ord[i]];
  if (e->d_items) cudaFree(e->d_items);
  e->d_items = nullptr;
  e->n_items = (int)sorted.size();
  e->h_items = sorted;
  if (!sorted.empty()) {
    GD_CUDA(cudaMalloc(&e->d_items, sizeof(WorkItem) * sorted.size()));
    GD_CUDA(cudaMemcpy(e->d_items, sorted.data(), sizeof(WorkItem) * sorted.size(), cudaMemcpyHostToDevice));
  }
  return GD_OK;
}

size_t smem_for(const gd_ensemble *e, int warps, int kst, int stage = 1, int group = 1)
{
  return kernel_smem_bytes(stage ? e->Pmax : 0, kst, e->lig_slots, warps, e->precision, group);
}

// Pick the KDE staging, the grid and (if not given) the replicas per CTA.
int configure(gd_ensemble *e, TileConfig tc)
{
  // the split (latency) form exists for the FP32 atom-pair loop of the batched kernel
  if (e->precision == GD_PREC_FP64 || e->kernel == GD_KERNEL_PLAIN || tc.kpl % 2) tc.group = 1;
  if (tc.group != 1 && tc.group != 2 && tc.group != 4 && tc.group != 8)
    return fail(GD_E_INVALID, "warps per replica = %d (1, 2, 4 or 8)", tc.group);
  if (tc.warps_per_cta < 1 || tc.warps_per_cta * 32 > kMaxCtaThreads || tc.warps_per_cta % tc.group)
    return fail(GD_E_INVALID, "warps per CTA = %d outside [1, %d] or not a multiple of the %d warps per replica",
                tc.warps_per_cta, kMaxCtaThreads / 32, tc.group);
  // a pocket too large to stage is read through L1; KDE points that do not fit are read from global memory
  if (tc.stage && smem_for(e, tc.warps_per_cta, 0, 1, tc.group) > kSmemLimit) tc.stage = 0;
  // FP32 reads the KDE points through L1 (the shared memory left to L1 pays more than
  // staging them); FP64 stages them
  e->Kst = e->precision == GD_PREC_FP64 ? e->Kmax : 0;
  if (smem_for(e, tc.warps_per_cta, e->Kst, tc.stage, tc.group) > kSmemLimit) e->Kst = 0;
  const size_t smem = smem_for(e, tc.warps_per_cta, e->Kst, tc.stage, tc.group);
  if (smem > kSmemLimit)
    return fail(GD_E_CAPACITY, "%d replicas per CTA need %zu B of shared memory (limit %zu)", tc.warps_per_cta, smem,
                kSmemLimit);
  const int occ = kernel_occupancy(0, e->precision, tc, smem);
  if (occ < 1) return fail(GD_E_INVALID, "tile (warps %d, kpl %d, ab %d) cannot launch", tc.warps_per_cta, tc.kpl, tc.ab);
  int nsm = 0;
  GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
  e->tc = tc;
  e->smem = smem;
  if (e->gexec) {
    cudaGraphExecDestroy(e->gexec);
    e->gexec = nullptr;
  }
  GD_TRY(build_items(e));
  e->grid = std::max(1, std::min(e->n_items, occ * nsm));
  return GD_OK;
}

// Replicas per CTA from occupancy: fewest waves of work items, then most
// resident warps per SM.
// stage_opt: -1 chooses between staging the pocket and reading it through L1.
int choose_warps(gd_ensemble *e, TileConfig base, int stage_opt = -1)
{
  int nsm = 0;
  GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
  double best = 1e300;
  const int G = (e->precision == GD_PREC_FP64 || e->kernel == GD_KERNEL_PLAIN || base.kpl % 2) ? 1
                                                                                         : std::max(1, base.group);
  int best_w = std::max(8, G), best_stage = 1;
  for (int stage = 1; stage >= 0; --stage)
  for (int w = std::max(2, G); w <= kMaxCtaThreads / 32; w += (w < G ? 1 : G)) {
    if (stage_opt >= 0 && stage != stage_opt) continue;
    if (w % G) continue;
    TileConfig tc = base;
    tc.warps_per_cta = w;
    tc.stage = stage;
    tc.group = G;
    int kst = e->Kmax;
    if (smem_for(e, w, kst, stage, G) > kSmemLimit) kst = 0;
    const size_t smem = smem_for(e, w, kst, stage, G);
    if (smem > kSmemLimit) continue;
    const int occ = kernel_occupancy(0, e->precision, tc, smem);
    if (occ < 1) continue;
    // items and the slowest SM's load (items are equal-cost within a job)
    long long items = 0;
    for (size_t j = 0; j < e->jobs.size(); ++j) {
      const std::vector<int> &pr = e->rep_prt[j];
      int r = 0;
      while (r < (int)pr.size()) {
        int k = 1;
        while (r + k < (int)pr.size() && k < w / G && pr[r + k] == pr[r]) ++k;
        ++items;
        r += k;
      }
    }
    const long long slots = (long long)occ * nsm;
    const long long waves = (items + slots - 1) / slots;
    // time ~ waves * (warps resident per SM); fewer resident warps per SM than 16 also hurts latency hiding
    const int resident = occ * w;
    double t = (double)waves * std::max(resident, 16) / (double)std::min(resident, 32);
    if (!stage) t *= 1.05;  // L1 reads of the pocket: prefer staging when occupancy is equal
    if (t < best - 1e-9) {
      best = t;
      best_w = w;
      best_stage = stage;
    }
  }
  TileConfig tc = base;
  tc.warps_per_cta = best_w;
  tc.stage = best_stage;
  tc.group = G;
  return configure(e, tc);
}

int upload_jobs(gd_ensemble *e)
{
  std::vector<DevJob> h(e->jobs.size());
  for (size_t j = 0; j < e->jobs.size(); ++j) h[j] = e->jobs[j].dj;
  if (e->d_jobs) cudaFree(e->d_jobs);
  GD_CUDA(cudaMalloc(&e->d_jobs, sizeof(DevJob) * std::max<size_t>(h.size(), 1)));
  GD_CUDA(cudaMemcpy(e->d_jobs, h.data(), sizeof(DevJob) * h.size(), cudaMemcpyHostToDevice));
  return GD_OK;
}

int finish_create(gd_ensemble *e)
{
  e->Pmax = 0;
  e->Kmax = 0;
  int Lmax = 1;
  e->rep_prt.resize(e->jobs.size());
  for (size_t j = 0; j < e->jobs.size(); ++j) {
    const DevJob &J = e->jobs[j].dj;
    e->Pmax = std::max(e->Pmax, J.npoint_pad);
    e->Kmax = std::max(e->Kmax, J.nkde);
    Lmax = std::max(Lmax, J.natom);
  }
  e->lig_slots = (Lmax + 3) & ~3;
  GD_TRY(upload_jobs(e));
  {
    const size_t nj = e->jobs.size();
    std::vector<int> xoff(2 * (nj + 1), 0);
    for (int par = 0; par < 2; ++par)
      for (size_t j = 0; j < nj; ++j) {
        const DevJob &J = e->jobs[j].dj;
        const int np = J.ntmp >= 2 ? (J.ntmp - par) / 2 : 0;
        xoff[par * (nj + 1) + j + 1] = xoff[par * (nj + 1) + j] + J.nprt * J.nlig * np;
      }
    e->xtot = std::max(xoff[nj], xoff[2 * (nj + 1) - 1]);
    GD_CUDA(cudaMalloc(&e->d_xoff, sizeof(int) * xoff.size()));
    GD_CUDA(cudaMemcpy(e->d_xoff, xoff.data(), sizeof(int) * xoff.size(), cudaMemcpyHostToDevice));
  }
  GD_CUDA(cudaMalloc(&e->d_step, sizeof(int)));
  GD_CUDA(cudaMalloc(&e->d_queue, sizeof(int)));
  // error words: [0] kernel flags (kErr*), [1..3] the device packer's failure details
  GD_CUDA(cudaMalloc(&e->d_err, 4 * sizeof(int)));
  GD_CUDA(cudaMemset(e->d_err, 0, 4 * sizeof(int)));
  GD_CUDA(cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking));
  const Options o = opts();
  e->kernel = o.kernel;
  e->precision = o.precision;
  e->use_graph = o.graph != 0;
  e->wait_limit = (uint32_t)o.wait_limit;
  e->stall_bytes = o.stall_test ? 16u : 0u;
  TileConfig tc{o.warps > 0 ? o.warps : 8, o.kpl, o.ab, o.stage != 0 ? 1 : 0, o.replica_warps};
  default_pair_tile(tc.group, tc.kpl, tc.ab);
  if (e->precision == GD_PREC_FP64) tc.kpl = 1, tc.ab = 8, tc.group = 1;
  if (o.warps > 0) return configure(e, tc);
  return choose_warps(e, tc, o.stage);
}

int read_replica_prt(gd_ensemble *e, size_t j, const std::vector<ReplicaMC> &reps)
{
  e->rep_prt[j].resize(reps.size());
  for (size_t r = 0; r < reps.size(); ++r) e->rep_prt[j][r] = reps[r].idx_prt;
  return GD_OK;
}

cudaEvent_t next_event(gd_ensemble *e)
{
  if (e->ev_used == (int)e->ev.size()) {
    cudaEvent_t x;
    if (cudaEventCreate(&x) != cudaSuccess) return nullptr;
    e->ev.push_back(x);
  }
  return e->ev[e->ev_used++];
}

int check_err(gd_ensemble *e)
{
  int h[4] = {0, 0, 0, 0};
  GD_CUDA(cudaMemcpy(h, e->d_err, sizeof(h), cudaMemcpyDeviceToHost));
  if (h[0] & kErrPack) {
    if (h[1] == kPackFailShape)
      return fail(GD_E_INVALID, "the Complex on the GPU differs in %s (%d) from the one the host described",
                  pack_field_name(h[2]), h[3]);
    return fail(h[1] == kPackFailCapacity ? GD_E_CAPACITY : GD_E_INVALID, "invalid Complex: %s: %d",
                pack_field_name(h[2]), h[3]);
  }
  if (h[0] & kErrTimeout) return fail(GD_E_TIMEOUT, "a bounded wait for a shared-memory bulk copy gave up");
  return GD_OK;
}

KArgs mc_args(gd_ensemble *e, int s_begin, int nsteps, int flags, const int *d_step);

int launch_mc(gd_ensemble *e, int s_begin, int nsteps, int flags)
{
  cudaEvent_t e0 = next_event(e), e1 = next_event(e);
  if (!e0 || !e1) return fail(GD_E_CUDA, "cudaEventCreate failed");
  GD_CUDA(cudaEventRecord(e0, e->st));
  if (e->kernel == GD_KERNEL_PLAIN) {
    for (size_t j = 0; j < e->jobs.size(); ++j)
      GD_CUDA(launch_plain(e->d_jobs + j, e->jobs[j].dj.nrep, s_begin, nsteps, flags, e->d_err, e->st));
    e->launches += (int)e->jobs.size();
    e->all_launches += (int)e->jobs.size();
  } else {
    GD_CUDA(cudaMemsetAsync(e->d_queue, 0, sizeof(int), e->st));
    GD_CUDA(launch_kernel(0, e->precision, e->tc, mc_args(e, s_begin, nsteps, flags, nullptr), e->grid, e->st));
    e->launches += 1;
    e->all_launches += 1;
  }
  GD_CUDA(cudaEventRecord(e1, e->st));
  return GD_OK;
}

KArgs mc_args(gd_ensemble *e, int s_begin, int nsteps, int flags, const int *d_step)
{
  KArgs a{};
  a.jobs = e->d_jobs;
  a.items = e->d_items;
  a.n_items = e->n_items;
  a.queue = e->d_queue;
  a.err = e->d_err;
  a.s_begin = s_begin;
  a.nsteps = nsteps;
  a.flags = flags;
  a.d_step = d_step;
  a.P = e->tc.stage ? e->Pmax : 0;
  a.Kst = e->Kst;
  a.lig_slots = e->lig_slots;
  a.group = (uint16_t)e->tc.group;
  a.wait_limit = e->wait_limit;
  a.stall_bytes = (uint16_t)e->stall_bytes;
  return a;
}

// One exchange interval (queue reset, Monte Carlo chunk of `chunk` steps from
// *d_step, exchange sweep, *d_step += chunk) captured once and replayed.
int interval_graph(gd_ensemble *e, int chunk)
{
  if (e->gexec && e->g_chunk == chunk) return GD_OK;
  if (e->gexec) {
    cudaGraphExecDestroy(e->gexec);
    e->gexec = nullptr;
  }
  cudaGraph_t g = nullptr;
  GD_CUDA(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaMemsetAsync(e->d_queue, 0, sizeof(int), e->st);
  if (ce == cudaSuccess) ce = launch_kernel(0, e->precision, e->tc, mc_args(e, 0, chunk, kMcStoreAccept, e->d_step), e->grid, e->st);
  if (ce == cudaSuccess)
    ce = launch_exchange_all(e->d_jobs, e->d_xoff, (int)e->jobs.size(), e->xtot, 0, e->d_step, chunk, chunk, e->st);
  if (ce == cudaSuccess) ce = launch_advance_step(e->d_step, chunk, e->st);
  const cudaError_t ee = cudaStreamEndCapture(e->st, &g);
  if (ce != cudaSuccess || ee != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return fail(GD_E_CUDA, "graph capture: %s", cudaGetErrorString(ce != cudaSuccess ? ce : ee));
  }
  ce = cudaGraphInstantiate(&e->gexec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) return fail(GD_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ce));
  e->g_chunk = chunk;
  return GD_OK;
}

int exchange_sweep(gd_ensemble *e, int x)
{
  if (e->xtot <= 0) return GD_OK;
  GD_CUDA(launch_exchange_all(e->d_jobs, e->d_xoff, (int)e->jobs.size(), e->xtot, x, nullptr, 0, 0, e->st));
  e->all_launches += 1;
  return GD_OK;
}

// nsteps steps from e->step, cut at exchange boundaries.  Whole exchange
// intervals of a plain run (no records) replay the captured interval graph.
int advance(gd_ensemble *e, int nsteps, int spx, int f_first, int f_all, int f_last)
{
  int done = 0;
  if (e->use_graph && e->kernel == GD_KERNEL_BATCHED && spx > 0 && f_first == 0 && f_all == 0 &&
      f_last == kMcStoreAccept && e->step % spx == 0 && nsteps >= spx) {
    const int n_int = nsteps / spx;
    if (interval_graph(e, spx) == GD_OK) {
      // a kernel argument rather than a copy from pageable memory, which
      // could wait for the stream
      GD_CUDA(launch_set_step(e->d_step, e->step, e->st));
      cudaEvent_t e0 = next_event(e), e1 = next_event(e);
      if (!e0 || !e1) return fail(GD_E_CUDA, "cudaEventCreate failed");
      GD_CUDA(cudaEventRecord(e0, e->st));
      for (int k = 0; k < n_int; ++k) GD_CUDA(cudaGraphLaunch(e->gexec, e->st));
      GD_CUDA(cudaEventRecord(e1, e->st));
      e->launches += n_int;
      e->all_launches += 1 + 3 * n_int;
      e->step += n_int * spx;
      done = n_int * spx;
    } else {
      e->use_graph = false;   // capture unavailable: launch chunk by chunk
    }
  }
  while (done < nsteps) {
    int chunk = nsteps - done;
    if (spx > 0) chunk = std::min(chunk, spx - (e->step % spx));
    const int f = f_all | (done == 0 ? f_first : 0) | (done + chunk == nsteps ? f_last : 0);
    GD_TRY(launch_mc(e, e->step, chunk, f));
    e->step += chunk;
    done += chunk;
    if (spx > 0 && e->step % spx == 0) GD_TRY(exchange_sweep(e, e->step / spx - 1));
  }
  return GD_OK;
}

void destroy(gd_ensemble *e)
{
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->st) cudaStreamSynchronize(e->st);
  for (auto &j : e->jobs) free_job(j);
  for (auto &p : e->pockets) free_pocket(p);
  if (e->d_jobs) cudaFree(e->d_jobs);
  if (e->d_items) cudaFree(e->d_items);
  if (e->d_queue) cudaFree(e->d_queue);
  if (e->d_err) cudaFree(e->d_err);
  if (e->d_xoff) cudaFree(e->d_xoff);
  if (e->d_step) cudaFree(e->d_step);
  if (e->gexec) cudaGraphExecDestroy(e->gexec);
  for (auto x : e->ev) cudaEventDestroy(x);
  if (e->st) cudaStreamDestroy(e->st);
  delete e;
}

// Ensemble of one job from a Complex replica range (the Dock path).
int ensemble_from_complex_range(const Complex *c, int rb, int re, uint64_t seed, Record *rec, int device,
                                gd_ensemble **out)
{
  *out = nullptr;
  Tracer tr("create");
  GD_TRY(set_device(device));
  PocketData pk;
  JobData jd;
  GD_TRY(pocket_from_complex(c, pk));
  GD_TRY(job_from_complex(c, rb, re, seed, jd));
  jd.cell_room = true;  // Dock refills this state in place from later Complexes
  tr.mark("read Complex");
  gd_ensemble *e = new gd_ensemble;
  e->device = device;
  e->pockets.resize(1);
  e->jobs.resize(1);
  int rc = pack_pocket(pk, e->pockets[0]);
  tr.mark("pack pocket");
  if (rc == GD_OK) rc = pack_job(jd, e->pockets[0], c->enepara, rec != nullptr, rec, e->jobs[0]);
  tr.mark("pack job");
  if (rc == GD_OK) {
    e->rep_prt.resize(1);
    read_replica_prt(e, 0, jd.reps);
    rc = finish_create(e);
  }
  tr.mark("configure");
  if (rc != GD_OK) {
    destroy(e);
    return rc;
  }
  *out = e;
  return GD_OK;
}

// The shapes Dock's cached state was packed for, read from a host Complex
// without packing it: true if `c` (replicas [rb, re]) has exactly these.
bool same_dock_shapes(const gd_ensemble *e, const Complex *c, int rb, int re)
{
  if (e->jobs.size() != 1 || e->pockets.size() != 1) return false;
  const DevJob &J = e->jobs[0].dj;
  const ComplexSize &sz = c->size;
  if (sz.n_prt < 1 || sz.n_prt > GD_MAX_CONF_PRT || sz.n_lig < 1 || sz.n_lig > GD_MAX_CONF_LIG ||
      sz.kde_npoint < 0 || sz.kde_npoint > GD_MAXKDE || sz.n_rep > GD_MAX_REP || rb < 0 || re >= sz.n_rep || rb > re)
    return false;
  int P = 0;
  for (int i = 0; i < sz.n_prt; ++i) P = std::max(P, c->prt[i].prt_npoint);
  const int Ppad = ((P + kPointAlign - 1) / kPointAlign) * kPointAlign;
  int nk = 0;
  for (int k = 0; k < sz.kde_npoint; ++k) nk += c->kde.t[k] >= 0 && c->kde.t[k] < kLigTypes;
  if (J.natom != c->lig[0].lig_natom || J.nlig != sz.n_lig || J.nprt != sz.n_prt || J.ntmp != sz.n_tmp ||
      J.nmcs != sz.mcs_nrow || J.npoint_pad != Ppad || e->pockets[0].Ppad != Ppad || J.nkde != nk ||
      J.nrep != re - rb + 1 || J.rid_base != rb || J.nrep_total != sz.n_rep)
    return false;
  const std::vector<int> &prt = e->rep_prt[0];
  for (int r = rb; r <= re; ++r)
    if (c->replica[r].idx_prt != prt[r - rb]) return false;  // the work items group replicas by it
  return true;
}

// Refill of Dock's cached state on the GPU: the device packer reads the
// Complex that CopyH2D put at d_cx and writes the arenas the state already
// holds (no host packing, no copy of packed arrays).  A Complex the packer
// refuses sets the ensemble's error flag, which the kernels and check_err see.
int dock_refill_device(gd_ensemble *e, const Complex *d_cx, int rb, int re, int n_rep, uint64_t seed, Record *rec)
{
  const DevJob &J = e->jobs[0].dj;
  const DevPocket &pk = e->pockets[0];
  PackDst D{};
  D.job = e->d_jobs;
  D.par = const_cast<DevParams *>(J.par);
  D.ref4 = const_cast<float4 *>(J.ref4);
  D.err = e->d_err;
  D.lgrp = const_cast<int2 *>(J.lgrp);
  D.lcenter = const_cast<float *>(J.lcenter);
  D.pcenter = pk.center;
  D.tcc = const_cast<float *>(J.tcc);
  D.lig = const_cast<float4 *>(J.lig);
  D.kde = const_cast<float4 *>(J.kde);
  D.mcs = const_cast<float4 *>(J.mcs);
  D.pos = pk.pos;
  D.aux = pk.aux;
  D.ncdc = pk.ncdc;
  D.psp = const_cast<float *>(J.psp);
  D.pspmask = const_cast<uint32_t *>(J.pspmask);
  D.pcell = const_cast<int4 *>(J.pcell);
  D.pcell_cnt = const_cast<int *>(J.pcell_cnt);
  D.pcell_stride = J.pcell_stride;
  D.kslot = const_cast<int4 *>(J.kslot);
  D.kde_cap = std::max(J.nkde, 1);
  D.Ppad = pk.Ppad;
  D.nkde_expect = J.nkde;
  D.expect_L = J.natom;
  D.expect_nlig = J.nlig;
  D.expect_nprt = J.nprt;
  D.expect_M = J.nmcs;
  D.expect_ntmp = J.ntmp;
  D.rep = J.rep;
  D.run_acc = J.run_acc;
  D.stats = J.stats;
  D.minus_beta = const_cast<float *>(J.minus_beta);
  D.rec = rec;
  D.rep_begin = rb;
  D.nrep = re - rb + 1;
  D.nrep_total = n_rep;
  D.key0 = (uint32_t)seed;
  D.key1 = (uint32_t)(seed >> 32);
  GD_CUDA(cudaMemsetAsync(e->d_err, 0, 4 * sizeof(int), e->st));
  GD_CUDA(device_pack(d_cx, D, e->st));
  e->all_launches += 3;
  e->jobs[0].dj.key0 = D.key0;  // the host copy of the header follows the device one
  e->jobs[0].dj.key1 = D.key1;
  e->jobs[0].dj.rec = rec;
  return GD_OK;
}

// Dock's ensemble on GPU `device`: the handle's cached one refilled in place
// when the shapes are unchanged (no allocation and no reconfiguration), by the
// device packer from the Complex CopyH2D put on the GPU (d_cx; option
// dock_device_pack) or else by the host packer (the packed pocket kept when
// the protein bytes are unchanged); otherwise a new one, which the handle
// then keeps.
int dock_ensemble(gd_rng *h, const Complex *c, const Complex *d_cx, int rb, int re, uint64_t seed, Record *rec,
                  int device, gd_ensemble **out)
{
  *out = nullptr;
  const Options o = opts();
  const size_t prt_bytes = sizeof(Protein) * (size_t)std::max(0, std::min(c->size.n_prt, GD_MAX_CONF_PRT));
  gd_ensemble *e = h->dock;
  ++h->dock_calls;
  if (e && e->device == device && same_options(h->dock_opt, o) && o.dock_device_pack && d_cx &&
      same_dock_shapes(e, c, rb, re)) {
    Tracer tr("refill on the GPU");
    GD_TRY(set_device(device));
    GD_CUDA(cudaStreamSynchronize(e->st));
    e->step = 0;
    e->ev_used = 0;
    e->launches = 0;
    e->all_launches = 0;
    GD_TRY(dock_refill_device(e, d_cx, rb, re, c->size.n_rep, seed, rec));
    h->dock_prt.clear();  // the host packer's record of the packed protein no longer holds
    tr.mark("pack enqueued");
    ++h->dock_reused;
    *out = e;
    return GD_OK;
  }
  if (e && e->device == device && same_options(h->dock_opt, o) && e->jobs.size() == 1) {
    Tracer tr("refill");
    GD_TRY(set_device(device));
    GD_CUDA(cudaStreamSynchronize(e->st));
    JobData jd;
    GD_TRY(job_from_complex(c, rb, re, seed, jd));
    jd.cell_room = true;  // the arena keeps the size of the one it refills
    bool ok = true;
    const bool same_prt = h->dock_prt.size() == prt_bytes &&
                          std::memcmp(h->dock_prt.data(), c->prt, prt_bytes) == 0 &&
                          e->pockets[0].hdb_types == hdb_point_types(c->enepara);
    if (!same_prt) {
      PocketData pk;
      GD_TRY(pocket_from_complex(c, pk));
      DevPocket np;
      GD_TRY(pack_pocket(pk, np, &e->pockets[0], e->st));
      if (np.arena != e->pockets[0].arena) {
        free_pocket(np);
        ok = false;
      } else {
        e->pockets[0] = np;
        h->dock_prt.assign((const unsigned char *)c->prt, (const unsigned char *)c->prt + prt_bytes);
      }
    }
    tr.mark("pocket");
    if (ok) {
      DevJobBuf nj;
      GD_TRY(pack_job(jd, e->pockets[0], c->enepara, rec != nullptr, rec, nj, &e->jobs[0], e->st));
      const DevJob &A = e->jobs[0].dj, &B = nj.dj;
      if (nj.arena != e->jobs[0].arena) {
        free_job(nj);
        ok = false;
      } else {
        ok = A.natom == B.natom && A.nlig == B.nlig && A.nprt == B.nprt && A.ntmp == B.ntmp && A.nrep == B.nrep &&
             A.nkde == B.nkde && A.nmcs == B.nmcs && A.npoint_pad == B.npoint_pad;
        e->jobs[0] = nj;
        std::vector<int> prt_of(jd.reps.size());
        for (size_t r = 0; r < jd.reps.size(); ++r) prt_of[r] = jd.reps[r].idx_prt;
        ok = ok && prt_of == e->rep_prt[0];
      }
    }
    tr.mark("job");
    if (ok) {
      GD_CUDA(cudaMemcpyAsync(e->d_jobs, &e->jobs[0].dj, sizeof(DevJob), cudaMemcpyHostToDevice, e->st));
      GD_CUDA(cudaMemsetAsync(e->d_err, 0, sizeof(int), e->st));
      e->step = 0;
      e->ev_used = 0;
      e->launches = 0;
      e->all_launches = 0;
      ++h->dock_reused;
      *out = e;
      return GD_OK;
    }
    destroy(e);  // shapes changed: a new ensemble below
    h->dock = nullptr;
    h->dock_prt.clear();
  } else if (e) {
    destroy(e);
    h->dock = nullptr;
    h->dock_prt.clear();
  }
  GD_TRY(ensemble_from_complex_range(c, rb, re, seed, rec, device, &e));
  if (!o.dock_cache) {  // the caller destroys it after the call
    *out = e;
    return GD_OK;
  }
  h->dock = e;
  h->dock_prt.assign((const unsigned char *)c->prt, (const unsigned char *)c->prt + prt_bytes);
  h->dock_opt = o;
  *out = e;
  return GD_OK;
}

}  // namespace

// =================================================================== C ABI
extern "C" {

int gd_set_ngpu(int n)
{
  if (n < 1) return fail(GD_E_INVALID, "ngpu = %d", n);
  std::lock_guard<std::mutex> lk(g_mu);
  g_ngpu = n;
  return GD_OK;
}

int gd_get_ngpu(void) { return ngpu(); }

int gd_set_option(const char *name, long long v)
{
  if (!name) return fail(GD_E_INVALID, "null option name");
  std::lock_guard<std::mutex> lk(g_mu);
  const std::string n(name);
  if (n == "kernel") {
    if (v != GD_KERNEL_BATCHED && v != GD_KERNEL_PLAIN) return fail(GD_E_INVALID, "kernel = %lld", v);
    g_opt.kernel = (int)v;
  } else if (n == "precision") {
    if (v < GD_PREC_FP32 || v > GD_PREC_FP64) return fail(GD_E_INVALID, "precision = %lld", v);
    g_opt.precision = (int)v;
  } else if (n == "warps") {
    if (v < 0 || v > kMaxCtaThreads / 32) return fail(GD_E_INVALID, "warps = %lld", v);
    g_opt.warps = (int)v;
  } else if (n == "kpl") {
    if (v != 0 && v != 1 && v != 2 && v != 4) return fail(GD_E_INVALID, "kpl = %lld", v);
    g_opt.kpl = (int)v;
  } else if (n == "ab") {
    if (v != 0 && v != 4 && v != 8) return fail(GD_E_INVALID, "ab = %lld", v);
    g_opt.ab = (int)v;
  } else if (n == "stage") {
    if (v < -1 || v > 1) return fail(GD_E_INVALID, "stage = %lld", v);
    g_opt.stage = (int)v;
  } else if (n == "dock_cache") {
    if (v != 0 && v != 1) return fail(GD_E_INVALID, "dock_cache = %lld", v);
    g_opt.dock_cache = (int)v;
  } else if (n == "replica_warps") {
    if (v != 1 && v != 2 && v != 4 && v != 8) return fail(GD_E_INVALID, "replica_warps = %lld (1, 2, 4 or 8)", v);
    g_opt.replica_warps = (int)v;
  } else if (n == "dock_device_pack") {
    if (v != 0 && v != 1) return fail(GD_E_INVALID, "dock_device_pack = %lld", v);
    g_opt.dock_device_pack = (int)v;
  } else if (n == "dock_record_direct") {
    if (v != 0 && v != 1) return fail(GD_E_INVALID, "dock_record_direct = %lld", v);
    g_opt.dock_record_direct = (int)v;
  } else if (n == "device_base") {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) count = 0;
    if (v < 0 || (count > 0 && v >= count)) return fail(GD_E_INVALID, "device_base = %lld (%d devices)", v, count);
    g_opt.device_base = (int)v;
  } else if (n == "wait_limit") {
    if (v < 0 || v > 0xffffffffLL) return fail(GD_E_INVALID, "wait_limit = %lld", v);
    g_opt.wait_limit = v;
  } else if (n == "stall_test") {
    if (v != 0 && v != 1) return fail(GD_E_INVALID, "stall_test = %lld", v);
    g_opt.stall_test = (int)v;
  } else if (n == "fail_alloc") {
    if (v < 0 || v > 1000000) return fail(GD_E_INVALID, "fail_alloc = %lld", v);
    set_injected_alloc_failures((int)v);
  } else if (n == "graph") {
    if (v != 0 && v != 1) return fail(GD_E_INVALID, "graph = %lld", v);
    g_opt.graph = (int)v;
  } else {
    return fail(GD_E_INVALID, "unknown option '%s'", name);
  }
  return GD_OK;
}

long long gd_get_option(const char *name)
{
  if (!name) return GD_E_INVALID;
  std::lock_guard<std::mutex> lk(g_mu);
  const std::string n(name);
  if (n == "kernel") return g_opt.kernel;
  if (n == "precision") return g_opt.precision;
  if (n == "warps") return g_opt.warps;
  if (n == "kpl") return g_opt.kpl;
  if (n == "ab") return g_opt.ab;
  if (n == "graph") return g_opt.graph;
  if (n == "stage") return g_opt.stage;
  if (n == "replica_warps") return g_opt.replica_warps;
  if (n == "dock_device_pack") return g_opt.dock_device_pack;
  if (n == "dock_record_direct") return g_opt.dock_record_direct;
  if (n == "dock_cache") return g_opt.dock_cache;
  if (n == "wait_limit") return g_opt.wait_limit;
  if (n == "device_base") return g_opt.device_base;
  if (n == "stall_test") return g_opt.stall_test;
  if (n == "fail_alloc") return injected_alloc_failures();
  return GD_E_INVALID;
}

// ---------------------------------------------------------------- Dock --
int SetDevice(void)
{
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) return fail(GD_E_NODEVICE, "no CUDA device");
  const int n = ngpu();
  if (dev_of(n - 1) >= count)
    return fail(GD_E_NODEVICE, "%d GPUs from device %d requested, %d present", n, dev_of(0), count);
  for (int g = 0; g < n; ++g) {
    GD_CUDA(cudaSetDevice(dev_of(g)));
    GD_CUDA(cudaDeviceSetCacheConfig(cudaFuncCachePreferShared));  // prepair.C:11-20
  }
  return GD_OK;
}

int DeviceAlloc(Complex **cd, Record **rd, gd_rng_t **rng)
{
  if (!cd || !rd || !rng) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  for (int g = 0; g < n; ++g) {
    GD_CUDA(cudaSetDevice(dev_of(g)));
    cd[g] = nullptr;
    rd[g] = nullptr;
    if (cudaMalloc((void **)&cd[g], sizeof(Complex)) != cudaSuccess)
      return fail(GD_E_NOMEM, "device Complex (%zu B) on GPU %d", sizeof(Complex), g);
    if (cudaMalloc((void **)&rd[g], sizeof(Record) * (size_t)GD_MAX_REP) != cudaSuccess)
      return fail(GD_E_NOMEM, "device Record[%d] on GPU %d", GD_MAX_REP, g);
    rng[g] = new gd_rng;
  }
  return GD_OK;
}

int DeviceFree(Complex **cd, Record **rd, gd_rng_t **rng)
{
  if (!cd || !rd || !rng) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  for (int g = 0; g < n; ++g) {
    GD_CUDA(cudaSetDevice(dev_of(g)));
    if (rng[g] && rng[g]->dock) destroy(rng[g]->dock);
    if (cd[g]) GD_CUDA(cudaFree(cd[g]));
    if (rd[g]) GD_CUDA(cudaFree(rd[g]));
    delete rng[g];
    cd[g] = nullptr;
    rd[g] = nullptr;
    rng[g] = nullptr;
  }
  return GD_OK;
}

// Replicas per GPU of the split of prepair.C:366-392 (maximising balance);
// with replica exchange on, cut at protein-conformation blocks so that exchange
// partners (same protein and ligand conformation) stay on one GPU.
static int split_per_gpu(const Complex *ch, int n, int *per_out)
{
  const int n_rep = ch->size.n_rep;
  if (n < 1) return fail(GD_E_INVALID, "ngpu = %d", n);
  if (n_rep < 1 || n_rep > GD_MAX_REP) return fail(GD_E_INVALID, "n_rep = %d", n_rep);
  int per = (n_rep + n - 1) / n;
  const McPara &mp = ch->mcpara;
  const bool exch = mp.steps_per_exchange > 0 && ch->size.n_tmp > 1;
  if (exch && n > 1) {
    const int block = ch->size.n_tmp * ch->size.n_lig;
    per = ((ch->size.n_prt + n - 1) / n) * block;
  }
  const int n_active = (n_rep + per - 1) / per;
  if (n_active < n) return fail(GD_E_INVALID, "%d replicas cannot keep %d GPUs busy", n_rep, n);
  *per_out = per;
  return GD_OK;
}

int SetParaT(Complex *ch, ParaT **pt)
{
  if (!ch || !pt) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  const int n_rep = ch->size.n_rep;
  int per = 0;
  GD_TRY(split_per_gpu(ch, n, &per));
  for (int g = 0; g < n; ++g) {
    pt[g]->rep_begin = per * g;
    pt[g]->rep_end = std::min(pt[g]->rep_begin + per, n_rep) - 1;
    pt[g]->n_rep = pt[g]->rep_end - pt[g]->rep_begin + 1;
    pt[g]->record_sz = (int)sizeof(Record) * pt[g]->n_rep;
  }
  return GD_OK;
}

int gd_replica_range(const Complex *ch, int ngpu, int g, int *rep_begin, int *rep_end)
{
  if (!ch || !rep_begin || !rep_end) return fail(GD_E_INVALID, "null argument");
  if (g < 0 || g >= ngpu) return fail(GD_E_INVALID, "GPU %d of %d", g, ngpu);
  int per = 0;
  GD_TRY(split_per_gpu(ch, ngpu, &per));
  *rep_begin = per * g;
  *rep_end = std::min(*rep_begin + per, ch->size.n_rep) - 1;
  return GD_OK;
}

int gd_ensemble_create_complex_range(const Complex *cx, int rep_begin, int rep_end, uint64_t seed, int device,
                                     gd_ensemble_t **out)
{
  if (!out || !cx) return fail(GD_E_INVALID, "null argument");
  *out = nullptr;
  if (rep_begin < 0 || rep_end < rep_begin || rep_end >= cx->size.n_rep)
    return fail(GD_E_INVALID, "replica range [%d, %d] of %d", rep_begin, rep_end, cx->size.n_rep);
  gd_ensemble *e = nullptr;
  GD_TRY(ensemble_from_complex_range(cx, rep_begin, rep_end, seed, nullptr, device, &e));
  *out = e;
  return GD_OK;
}

int CopyH2D(Complex *ch, Complex **cd, ParaT **pt)
{
  if (!ch || !cd || !pt) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  for (int g = 0; g < n; ++g) {
    GD_CUDA(cudaSetDevice(dev_of(g)));
    ch->rep_begin = pt[g]->rep_begin;  // prepair.C:119-123
    ch->rep_end = pt[g]->rep_end;
    GD_CUDA(cudaMemcpy(cd[g], ch, sizeof(Complex), cudaMemcpyHostToDevice));
  }
  return GD_OK;
}

int InitCurand(gd_rng_t **rng)
{
  if (!rng) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  const char *env = std::getenv("GDOCK_SEED");
  const uint64_t base = env ? std::strtoull(env, nullptr, 10) : (uint64_t)std::time(nullptr);
  for (int g = 0; g < n; ++g) {
    if (!rng[g]) return fail(GD_E_STATE, "InitCurand before DeviceAlloc");
    if (!rng[g]->seeded) {
      rng[g]->seed = base + (uint64_t)g;  // backend_gpu.cu:52-56: one seed per GPU
      rng[g]->seeded = 1;
    }
    rng[g]->calls = 0;
  }
  return GD_OK;
}

int gd_rng_dock_reuse(const gd_rng_t *rng, uint64_t *calls, uint64_t *reused)
{
  if (!rng || !calls || !reused) return fail(GD_E_INVALID, "null argument");
  *calls = rng->dock_calls;
  *reused = rng->dock_reused;
  return GD_OK;
}

int gd_rng_seed(gd_rng_t *rng, uint64_t seed)
{
  if (!rng) return fail(GD_E_INVALID, "null rng");
  rng->seed = seed;
  rng->seeded = 1;
  rng->calls = 0;
  return GD_OK;
}

int Dock(Complex *ch, Record *rh, Complex **cd, Record **rd, ParaT **pt, gd_rng_t **rng)
{
  if (!ch || !rh || !cd || !rd || !pt || !rng) return fail(GD_E_INVALID, "null argument");
  const int n = ngpu();
  const McPara &mp = ch->mcpara;
  const int steps_total = mp.steps_total, spd = mp.steps_per_dump;
  if (steps_total < 0) return fail(GD_E_INVALID, "steps_total = %d", steps_total);
  if (spd < 1 || spd > GD_STEPS_PER_DUMP)
    return fail(GD_E_INVALID, "steps_per_dump = %d outside [1, %d] (Record capacity)", spd, GD_STEPS_PER_DUMP);
  const int spx = (mp.steps_per_exchange > 0 && ch->size.n_tmp > 1) ? mp.steps_per_exchange : 0;
  std::vector<gd_ensemble *> ens(n, nullptr);
  // where the kernels write the Records: the device array rd[g], copied to rh after each
  // chunk (backend_gpu.cu:108-110), or, when rh is page-locked host memory this GPU can
  // address (cudaHostAlloc, or cudaHostRegister with mapping), rh itself: each entry then
  // crosses PCIe as the kernel writes it, while the chunk runs, and no copy follows
  std::vector<Record *> rdst(n, nullptr);
  std::vector<char> direct(n, 0);
  const bool try_direct = opts().dock_record_direct != 0;
  int rc = GD_OK;
  Tracer tr("Dock");
  for (int g = 0; g < n && rc == GD_OK; ++g) {
    if (!rng[g] || !cd[g] || !rd[g]) {
      rc = fail(GD_E_STATE, "Dock before DeviceAlloc/InitCurand on GPU %d", g);
      break;
    }
    rdst[g] = rd[g];
    if (try_direct && (rc = set_device(dev_of(g))) == GD_OK) {
      cudaPointerAttributes at{};
      if (cudaPointerGetAttributes(&at, rh + pt[g]->rep_begin) == cudaSuccess && at.type == cudaMemoryTypeHost &&
          at.devicePointer != nullptr) {
        rdst[g] = (Record *)at.devicePointer;
        direct[g] = 1;
      } else {
        (void)cudaGetLastError();  // pageable memory: the copy below
      }
    }
    if (rc != GD_OK) break;
    // each Dock call draws a fresh stream from the handle (the reference's curand state advances)
    const uint64_t seed = rng[g]->seed + (rng[g]->calls++ << 32);
    rc = dock_ensemble(rng[g], ch, cd[g], pt[g]->rep_begin, pt[g]->rep_end, seed, rdst[g], dev_of(g), &ens[g]);
  }
  tr.mark("pack+create");
  // initial energy, backend_gpu.cu:87-91: one step, no move, forced accept
  for (int g = 0; g < n && rc == GD_OK; ++g) {
    rc = set_device(dev_of(g));
    if (rc == GD_OK) rc = launch_mc(ens[g], 0, 1, kMcInitial | kMcRecord | kMcResetRecord | kMcStoreAccept);
  }
  tr.mark("initial (enqueued)");
  // dump chunks, backend_gpu.cu:96-114
  for (int s1 = 0; s1 < steps_total && rc == GD_OK; s1 += spd) {
    for (int g = 0; g < n && rc == GD_OK; ++g) {
      rc = set_device(dev_of(g));
      ens[g]->step = s1;
      if (rc == GD_OK) rc = advance(ens[g], spd, spx, kMcResetRecord, kMcRecord, kMcStoreAccept);
    }
    for (int g = 0; g < n && rc == GD_OK; ++g) {
      rc = set_device(dev_of(g));
      if (rc != GD_OK) break;
      const cudaError_t ce =
          direct[g] ? cudaSuccess
                    : cudaMemcpyAsync(rh + pt[g]->rep_begin, rd[g], sizeof(Record) * (size_t)pt[g]->n_rep,
                                      cudaMemcpyDeviceToHost, ens[g]->st);
      if (ce == cudaSuccess) {
        const cudaError_t se = cudaStreamSynchronize(ens[g]->st);
        if (se != cudaSuccess) rc = fail(GD_E_CUDA, "Dock: %s", cudaGetErrorString(se));
      } else {
        rc = fail(GD_E_CUDA, "Dock record copy: %s", cudaGetErrorString(ce));
      }
      if (rc == GD_OK) rc = check_err(ens[g]);
    }
    tr.mark("chunk + record copy");
  }
  // final replica states: device Complex (as the reference) and the host Complex
  for (int g = 0; g < n && rc == GD_OK; ++g) {
    rc = set_device(dev_of(g));
    if (rc != GD_OK) break;
    const DevJob &J = ens[g]->jobs[0].dj;
    const size_t bytes = sizeof(ReplicaMC) * (size_t)J.nrep;
    if (cudaMemcpyAsync(cd[g]->replica + pt[g]->rep_begin, J.rep, bytes, cudaMemcpyDeviceToDevice, ens[g]->st) !=
            cudaSuccess ||
        cudaMemcpyAsync(ch->replica + pt[g]->rep_begin, J.rep, bytes, cudaMemcpyDeviceToHost, ens[g]->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(ens[g]->st) != cudaSuccess)
      rc = fail(GD_E_CUDA, "Dock final copy on GPU %d", g);
  }
  tr.mark("final replica copy");
  for (int g = 0; g < n; ++g)
    if (ens[g] && (!rng[g] || rng[g]->dock != ens[g])) destroy(ens[g]);  // not cached
  if (rc != GD_OK)
    for (int g = 0; g < n; ++g)
      if (rng[g] && rng[g]->dock) {  // drop the cached state of a failed call
        destroy(rng[g]->dock);
        rng[g]->dock = nullptr;
        rng[g]->dock_prt.clear();
      }
  return rc;
}

// ------------------------------------------------------------ poses --
// Energies of n poses of job `job` of a resident ensemble (mode 1 of the
// batched kernel): poses grouped by protein conformation, one warp per pose.
int eval_on(gd_ensemble *e, int job, int n, const int *conf, const float *mm, int precision, float *out,
            double *out64, float *raw)
{
  const DevJob &J = e->jobs[job].dj;
  for (int i = 0; i < n; ++i)
    if (conf[2 * i] < 0 || conf[2 * i] >= J.nlig || conf[2 * i + 1] < 0 || conf[2 * i + 1] >= J.nprt)
      return fail(GD_E_INVALID, "pose %d: conformation (%d, %d) out of range", i, conf[2 * i], conf[2 * i + 1]);
  const Options o = opts();
  TileConfig tc{8, o.kpl, o.ab};
  default_pair_tile(1, tc.kpl, tc.ab);
  if (precision == GD_PREC_FP64) tc.kpl = 1, tc.ab = 8;
  int kst = precision == GD_PREC_FP64 ? J.nkde : 0;  // FP32: KDE points through L1
  int P = e->Pmax;
  if (kernel_smem_bytes(P, 0, e->lig_slots, tc.warps_per_cta, precision) > kSmemLimit) P = 0;  // through L1
  size_t smem = kernel_smem_bytes(P, kst, e->lig_slots, tc.warps_per_cta, precision);
  if (smem > kSmemLimit) {
    kst = 0;
    smem = kernel_smem_bytes(P, kst, e->lig_slots, tc.warps_per_cta, precision);
  }
  if (smem > kSmemLimit) return fail(GD_E_CAPACITY, "ligand slots too large for shared memory");
  // poses grouped by protein conformation so that a CTA stages one conformation
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return conf[2 * a + 1] < conf[2 * b + 1]; });
  std::vector<int> sconf(2 * (size_t)n);
  std::vector<float> smm(6 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    sconf[2 * i] = conf[2 * ord[i]];
    sconf[2 * i + 1] = conf[2 * ord[i] + 1];
    for (int k = 0; k < 6; ++k) smm[6 * i + k] = mm[6 * (size_t)ord[i] + k];
  }
  std::vector<WorkItem> items;
  for (int i = 0; i < n;) {
    int k = 1;
    while (i + k < n && k < tc.warps_per_cta && sconf[2 * (i + k) + 1] == sconf[2 * i + 1]) ++k;
    items.push_back(WorkItem{job, sconf[2 * i + 1], i, k});
    i += k;
  }
  int *d_conf = nullptr;
  float *d_mm = nullptr, *d_out = nullptr, *d_raw = nullptr;
  double *d_out64 = nullptr;
  WorkItem *d_items = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_conf);
    cudaFree(d_mm);
    cudaFree(d_out);
    cudaFree(d_raw);
    cudaFree(d_out64);
    cudaFree(d_items);
  };
#define EV_CUDA(call)                                                                         \
  do {                                                                                        \
    cudaError_t ce_ = (call);                                                                 \
    if (ce_ != cudaSuccess) {                                                                 \
      cleanup();                                                                              \
      return fail(GD_E_CUDA, "pose evaluation: %s: %s", #call, cudaGetErrorString(ce_));      \
    }                                                                                         \
  } while (0)
  EV_CUDA(cudaMalloc(&d_conf, sizeof(int) * 2 * n));
  EV_CUDA(cudaMalloc(&d_mm, sizeof(float) * 6 * n));
  EV_CUDA(cudaMalloc(&d_out, sizeof(float) * 10 * n));
  if (raw) EV_CUDA(cudaMalloc(&d_raw, sizeof(float) * 9 * n));
  if (out64) EV_CUDA(cudaMalloc(&d_out64, sizeof(double) * 10 * n));
  EV_CUDA(cudaMalloc(&d_items, sizeof(WorkItem) * items.size()));
  EV_CUDA(cudaMemcpyAsync(d_conf, sconf.data(), sizeof(int) * 2 * n, cudaMemcpyHostToDevice, e->st));
  EV_CUDA(cudaMemcpyAsync(d_mm, smm.data(), sizeof(float) * 6 * n, cudaMemcpyHostToDevice, e->st));
  EV_CUDA(cudaMemcpyAsync(d_items, items.data(), sizeof(WorkItem) * items.size(), cudaMemcpyHostToDevice, e->st));
  EV_CUDA(cudaMemsetAsync(e->d_queue, 0, sizeof(int), e->st));
  KArgs a{};
  a.jobs = e->d_jobs;
  a.items = d_items;
  a.n_items = (int)items.size();
  a.queue = e->d_queue;
  a.err = e->d_err;
  a.P = P;
  a.Kst = kst;
  a.lig_slots = e->lig_slots;
  a.conf = d_conf;
  a.mm = d_mm;
  a.out = d_out;
  a.out64 = d_out64;
  a.raw = d_raw;
  int nsm = 0;
  EV_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, e->device));
  const int occ = std::max(1, kernel_occupancy(1, precision, tc, smem));
  const int grid = std::max(1, std::min((int)items.size(), occ * nsm));
  EV_CUDA(launch_kernel(1, precision, tc, a, grid, e->st));
  std::vector<float> hout(10 * (size_t)n), hraw(raw ? 9 * (size_t)n : 0);
  std::vector<double> hout64(out64 ? 10 * (size_t)n : 0);
  EV_CUDA(cudaMemcpyAsync(hout.data(), d_out, sizeof(float) * 10 * n, cudaMemcpyDeviceToHost, e->st));
  if (raw) EV_CUDA(cudaMemcpyAsync(hraw.data(), d_raw, sizeof(float) * 9 * n, cudaMemcpyDeviceToHost, e->st));
  if (out64) EV_CUDA(cudaMemcpyAsync(hout64.data(), d_out64, sizeof(double) * 10 * n, cudaMemcpyDeviceToHost, e->st));
  EV_CUDA(cudaStreamSynchronize(e->st));
#undef EV_CUDA
  for (int i = 0; i < n; ++i) {
    const size_t o2 = (size_t)ord[i];
    std::memcpy(out + 10 * o2, &hout[10 * (size_t)i], sizeof(float) * 10);
    if (raw) std::memcpy(raw + 9 * o2, &hraw[9 * (size_t)i], sizeof(float) * 9);
    if (out64) std::memcpy(out64 + 10 * o2, &hout64[10 * (size_t)i], sizeof(double) * 10);
  }
  cleanup();
  return check_err(e);
}

int gd_eval_poses(const Complex *c, int n, const int *conf, const float *mm, int precision, float *out,
                  double *out64, float *raw)
{
  if (!c || n < 0 || (n > 0 && (!conf || !mm || !out))) return fail(GD_E_INVALID, "null argument");
  if (precision < GD_PREC_FP32 || precision > GD_PREC_FP64) return fail(GD_E_INVALID, "precision = %d", precision);
  if (n == 0) return GD_OK;
  for (int i = 0; i < n; ++i)
    if (conf[2 * i] < 0 || conf[2 * i] >= c->size.n_lig || conf[2 * i + 1] < 0 || conf[2 * i + 1] >= c->size.n_prt)
      return fail(GD_E_INVALID, "pose %d: conformation (%d, %d) out of range", i, conf[2 * i], conf[2 * i + 1]);
  int dev = 0;
  GD_CUDA(cudaGetDevice(&dev));
  PocketData pk;
  JobData jd;
  GD_TRY(pocket_from_complex(c, pk));
  GD_TRY(job_from_complex(c, 0, 0, 0, jd));
  gd_ensemble *e = new gd_ensemble;
  e->device = dev;
  e->pockets.resize(1);
  e->jobs.resize(1);
  int rc = pack_pocket(pk, e->pockets[0]);
  if (rc == GD_OK) rc = pack_job(jd, e->pockets[0], c->enepara, false, nullptr, e->jobs[0]);
  if (rc == GD_OK) {
    const DevJob &J = e->jobs[0].dj;
    e->precision = precision;
    e->Pmax = J.npoint_pad;
    e->Kmax = J.nkde;
    e->lig_slots = (J.natom + 3) & ~3;
    rc = upload_jobs(e);
  }
  if (rc == GD_OK && cudaMalloc(&e->d_queue, sizeof(int)) != cudaSuccess) rc = fail(GD_E_CUDA, "cudaMalloc");
  // error words as an ensemble's: kernel flags, then the device packer's details
  if (rc == GD_OK && cudaMalloc(&e->d_err, 4 * sizeof(int)) != cudaSuccess) rc = fail(GD_E_CUDA, "cudaMalloc");
  if (rc == GD_OK && cudaMemset(e->d_err, 0, 4 * sizeof(int)) != cudaSuccess) rc = fail(GD_E_CUDA, "cudaMemset");
  if (rc == GD_OK && cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) != cudaSuccess)
    rc = fail(GD_E_CUDA, "cudaStreamCreate");
  if (rc == GD_OK) rc = eval_on(e, 0, n, conf, mm, precision, out, out64, raw);
  destroy(e);
  return rc;
}

// ---------------------------------------------------------- ensembles --
int gd_ensemble_create(const gd_pocket_desc_t *pockets, int npocket, const gd_job_desc_t *jobs, int njob,
                       const EnePara *enepara, int device, gd_ensemble_t **out)
{
  if (!out) return fail(GD_E_INVALID, "null out");
  *out = nullptr;
  if (!pockets || npocket < 1 || !jobs || njob < 1 || !enepara) return fail(GD_E_INVALID, "empty ensemble");
  GD_TRY(set_device(device));
  gd_ensemble *e = new gd_ensemble;
  e->device = device;
  e->pockets.resize(npocket);
  e->jobs.resize(njob);
  e->rep_prt.resize(njob);
  int rc = GD_OK;
  std::vector<int> nconf(npocket);
  for (int p = 0; p < npocket && rc == GD_OK; ++p) {
    PocketData pk;
    rc = pocket_from_desc(pockets[p], pk);
    pk.hdb_types = hdb_point_types(*enepara);
    if (rc == GD_OK) rc = pack_pocket(pk, e->pockets[p]);
    nconf[p] = pockets[p].nconf;
  }
  for (int j = 0; j < njob && rc == GD_OK; ++j) {
    const int p = jobs[j].pocket;
    if (p < 0 || p >= npocket) {
      rc = fail(GD_E_INVALID, "job %d: pocket %d out of range", j, p);
      break;
    }
    JobData jd;
    rc = job_from_desc(jobs[j], nconf[p], jd);
    if (rc == GD_OK) rc = pack_job(jd, e->pockets[p], *enepara, false, nullptr, e->jobs[j]);
    if (rc == GD_OK) read_replica_prt(e, j, jd.reps);
    e->jobs[j].pocket = p;
  }
  if (rc == GD_OK) rc = finish_create(e);
  if (rc != GD_OK) {
    destroy(e);
    return rc;
  }
  *out = e;
  return GD_OK;
}

int gd_ensemble_create_complex(const Complex *const *cx, int n, const uint64_t *seeds, int device,
                               gd_ensemble_t **out)
{
  if (!out) return fail(GD_E_INVALID, "null out");
  *out = nullptr;
  if (!cx || n < 1) return fail(GD_E_INVALID, "empty ensemble");
  GD_TRY(set_device(device));
  gd_ensemble *e = new gd_ensemble;
  e->device = device;
  e->jobs.resize(n);
  e->rep_prt.resize(n);
  std::vector<PocketData> seen;
  int rc = GD_OK;
  for (int j = 0; j < n && rc == GD_OK; ++j) {
    PocketData pk;
    JobData jd;
    rc = pocket_from_complex(cx[j], pk);
    if (rc == GD_OK) rc = job_from_complex(cx[j], 0, cx[j]->size.n_rep - 1, seeds ? seeds[j] : 0, jd);
    if (rc != GD_OK) break;
    // identical protein conformation sets share one device pocket
    int p = -1;
    for (size_t q = 0; q < seen.size(); ++q)
      if (seen[q].nconf == pk.nconf && seen[q].npts == pk.npts && seen[q].xyz == pk.xyz && seen[q].type == pk.type &&
          seen[q].cls == pk.cls && seen[q].cdc == pk.cdc && seen[q].seq3r == pk.seq3r && seen[q].hpp == pk.hpp &&
          seen[q].ele == pk.ele && seen[q].center == pk.center && seen[q].hdb_types == pk.hdb_types) {
        p = (int)q;
        break;
      }
    if (p < 0) {
      e->pockets.emplace_back();
      rc = pack_pocket(pk, e->pockets.back());
      seen.push_back(std::move(pk));
      p = (int)seen.size() - 1;
    }
    if (rc == GD_OK) rc = pack_job(jd, e->pockets[p], cx[j]->enepara, false, nullptr, e->jobs[j]);
    if (rc == GD_OK) read_replica_prt(e, j, jd.reps);
    e->jobs[j].pocket = p;
  }
  if (rc == GD_OK) rc = finish_create(e);
  if (rc != GD_OK) {
    destroy(e);
    return rc;
  }
  *out = e;
  return GD_OK;
}

int gd_ensemble_init(gd_ensemble_t *e)
{
  if (!e) return fail(GD_E_INVALID, "null ensemble");
  GD_TRY(set_device(e->device));
  return launch_mc(e, 0, 1, kMcInitial | kMcStoreAccept);
}

int gd_ensemble_run(gd_ensemble_t *e, int nsteps, int steps_per_exchange)
{
  if (!e) return fail(GD_E_INVALID, "null ensemble");
  if (nsteps < 0 || steps_per_exchange < 0) return fail(GD_E_INVALID, "nsteps = %d, steps_per_exchange = %d", nsteps, steps_per_exchange);
  GD_TRY(set_device(e->device));
  return advance(e, nsteps, steps_per_exchange, 0, 0, kMcStoreAccept);
}

int gd_ensemble_sync(gd_ensemble_t *e, double *kernel_ms, int *launches, int *all_launches)
{
  if (!e) return fail(GD_E_INVALID, "null ensemble");
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  double ms = 0;
  for (int i = 0; i + 1 < e->ev_used; i += 2) {
    float t = 0;
    GD_CUDA(cudaEventElapsedTime(&t, e->ev[i], e->ev[i + 1]));
    ms += t;
  }
  if (kernel_ms) *kernel_ms = ms;
  if (launches) *launches = e->launches;
  if (all_launches) *all_launches = e->all_launches;
  e->ev_used = 0;
  e->launches = 0;
  e->all_launches = 0;
  return check_err(e);
}

int gd_ensemble_num_replicas(const gd_ensemble_t *e, int job)
{
  if (!e || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  return e->jobs[job].dj.nrep;
}

int gd_ensemble_replicas(gd_ensemble_t *e, int job, ReplicaMC *out)
{
  if (!e || !out || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  GD_TRY(set_device(e->device));
  const DevJob &J = e->jobs[job].dj;
  GD_CUDA(cudaMemcpyAsync(out, J.rep, sizeof(ReplicaMC) * (size_t)J.nrep, cudaMemcpyDeviceToHost, e->st));
  GD_CUDA(cudaStreamSynchronize(e->st));
  return GD_OK;
}

int gd_ensemble_best_poses(gd_ensemble_t *e, int job, float *best_mm, double *best_energy)
{
  if (!e || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  GD_TRY(set_device(e->device));
  const DevJob &J = e->jobs[job].dj;
  std::vector<RepStats> s(J.nrep);
  GD_CUDA(cudaMemcpyAsync(s.data(), J.stats, sizeof(RepStats) * s.size(), cudaMemcpyDeviceToHost, e->st));
  GD_CUDA(cudaStreamSynchronize(e->st));
  for (int r = 0; r < J.nrep; ++r) {
    if (best_mm)
      for (int k = 0; k < 6; ++k) best_mm[6 * (size_t)r + k] = s[r].best_mm[k];
    if (best_energy) best_energy[r] = s[r].best_e;
  }
  return GD_OK;
}

int gd_ensemble_cluster(gd_ensemble_t *e, int job, int ref_lig, const float *ref_mm, float rmsd_cut,
                        gd_cluster_t *clusters, int max_clusters, int *n_clusters, int *cluster_of,
                        float *rmsd_to_ref)
{
  if (!e || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  if (!n_clusters || (max_clusters > 0 && !clusters) || max_clusters < 0) return fail(GD_E_INVALID, "null argument");
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  return cluster_job(e->jobs[job].dj, e->d_jobs + job, e->st, ref_lig, ref_mm, rmsd_cut, clusters, max_clusters,
                     n_clusters, cluster_of, rmsd_to_ref);
}

int gd_ensemble_eval_poses(gd_ensemble_t *e, int job, int n, const int *conf, const float *mm, int precision,
                           float *out, double *out64, float *raw)
{
  if (!e || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  if (n < 0 || (n > 0 && (!conf || !mm || !out))) return fail(GD_E_INVALID, "null argument");
  if (precision < GD_PREC_FP32 || precision > GD_PREC_FP64) return fail(GD_E_INVALID, "precision = %d", precision);
  if (n == 0) return GD_OK;
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  return eval_on(e, job, n, conf, mm, precision, out, out64, raw);
}

int gd_ensemble_stats(gd_ensemble_t *e, int job, double *out8)
{
  if (!e || !out8 || job < 0 || job >= (int)e->jobs.size()) return fail(GD_E_INVALID, "job %d", job);
  GD_TRY(set_device(e->device));
  const DevJob &J = e->jobs[job].dj;
  std::vector<RepStats> s(J.nrep);
  GD_CUDA(cudaMemcpyAsync(s.data(), J.stats, sizeof(RepStats) * s.size(), cudaMemcpyDeviceToHost, e->st));
  GD_CUDA(cudaStreamSynchronize(e->st));
  for (int r = 0; r < J.nrep; ++r) {
    const RepStats &x = s[r];
    double *o = out8 + 8 * (size_t)r;
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
  return GD_OK;
}

int gd_ensemble_autotune(gd_ensemble_t *e, int steps, char *report, int report_len)
{
  if (!e || steps < 1) return fail(GD_E_INVALID, "autotune: steps = %d", steps);
  if (e->kernel != GD_KERNEL_BATCHED) return GD_OK;
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  // snapshot of everything a Monte Carlo launch writes (records are not written: no record flags)
  std::vector<void *> snaps;
  auto snap_bytes = [](const DevJob &J) {
    return sizeof(ReplicaMC) * (size_t)J.nrep + sizeof(int) * (size_t)J.nrep + sizeof(RepStats) * (size_t)J.nrep;
  };
  int rc = GD_OK;
  for (auto &jb : e->jobs) {
    void *p = nullptr;
    const DevJob &J = jb.dj;
    if (cudaMalloc(&p, snap_bytes(J)) != cudaSuccess) {
      rc = fail(GD_E_NOMEM, "autotune snapshot");
      break;
    }
    unsigned char *b = (unsigned char *)p;
    cudaMemcpyAsync(b, J.rep, sizeof(ReplicaMC) * J.nrep, cudaMemcpyDeviceToDevice, e->st);
    cudaMemcpyAsync(b + sizeof(ReplicaMC) * J.nrep, J.run_acc, sizeof(int) * J.nrep, cudaMemcpyDeviceToDevice, e->st);
    cudaMemcpyAsync(b + (sizeof(ReplicaMC) + sizeof(int)) * J.nrep, J.stats, sizeof(RepStats) * J.nrep,
                    cudaMemcpyDeviceToDevice, e->st);
    snaps.push_back(p);
  }
  auto restore = [&]() {
    for (size_t j = 0; j < e->jobs.size() && j < snaps.size(); ++j) {
      const DevJob &J = e->jobs[j].dj;
      unsigned char *b = (unsigned char *)snaps[j];
      cudaMemcpyAsync(J.rep, b, sizeof(ReplicaMC) * J.nrep, cudaMemcpyDeviceToDevice, e->st);
      cudaMemcpyAsync(J.run_acc, b + sizeof(ReplicaMC) * J.nrep, sizeof(int) * J.nrep, cudaMemcpyDeviceToDevice, e->st);
      cudaMemcpyAsync(J.stats, b + (sizeof(ReplicaMC) + sizeof(int)) * J.nrep, sizeof(RepStats) * J.nrep,
                      cudaMemcpyDeviceToDevice, e->st);
    }
  };
  std::string rep;
  TileConfig best = e->tc;
  double best_t = 1e300;
  const int shapes[][2] = {{1, 8}, {2, 4}, {2, 8}, {4, 4}, {4, 8}};
  const int warps[] = {4, 6, 8, 10, 12, 14, 16};
  const bool can_stage = smem_for(e, std::max(4, e->tc.group), 0, 1, e->tc.group) <= kSmemLimit;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  for (int stage = can_stage ? 1 : 0; stage >= 0; --stage)
  for (const auto &sh : shapes) {
    if (e->precision == GD_PREC_FP64 && !(sh[0] == 1 && sh[1] == 8)) continue;
    // FP32: kpl 1 is the per-type-group scalar loop, which the atom-pair loop of
    // the even kpl shapes outruns on every workload measured; not worth tuning time
    if (e->precision != GD_PREC_FP64 && sh[0] == 1) continue;
    for (int w : warps) {
      if (rc != GD_OK) break;
      // the warps per replica are kept; the candidates are the multiples of it
      if (w % e->tc.group) continue;
      TileConfig tc{w, sh[0], sh[1], stage, e->tc.group};
      if (configure(e, tc) != GD_OK || e->tc.stage != stage) continue;
      // a strided sample of the work items (heaviest-first order kept), about two
      // waves of the grid, so that a candidate runs the full chunk length
      const int stride = std::max(1, e->n_items / std::max(1, 2 * e->grid));
      std::vector<WorkItem> sample;
      for (int i = 0; i < e->n_items; i += stride) sample.push_back(e->h_items[i]);
      WorkItem *d_sample = nullptr;
      if (cudaMalloc(&d_sample, sizeof(WorkItem) * sample.size()) != cudaSuccess ||
          cudaMemcpyAsync(d_sample, sample.data(), sizeof(WorkItem) * sample.size(), cudaMemcpyHostToDevice,
                          e->st) != cudaSuccess) {
        cudaFree(d_sample);
        rc = fail(GD_E_CUDA, "autotune sample");
        break;
      }
      KArgs ka = mc_args(e, e->step, steps, 0, nullptr);
      ka.items = d_sample;
      ka.n_items = (int)sample.size();
      float t = 0;
      cudaMemsetAsync(e->d_queue, 0, sizeof(int), e->st);
      cudaEventRecord(a, e->st);
      const cudaError_t le = launch_kernel(0, e->precision, e->tc, ka, std::min(e->grid, ka.n_items), e->st);
      cudaEventRecord(b, e->st);
      if (le != cudaSuccess || cudaStreamSynchronize(e->st) != cudaSuccess) rc = fail(GD_E_CUDA, "autotune launch");
      cudaEventElapsedTime(&t, a, b);
      cudaFree(d_sample);
      restore();
      t *= (float)e->n_items / (float)sample.size();   // per whole launch
      char line[160];
      snprintf(line, sizeof line, "warps=%d kpl=%d ab=%d stage=%d grid=%d items=%d: %.3f ms\n", w, sh[0], sh[1],
               stage, e->grid, e->n_items, t);
      rep += line;
      if (t < best_t) {
        best_t = t;
        best = tc;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamSynchronize(e->st);
  for (void *p : snaps) cudaFree(p);
  e->ev_used = 0;
  e->launches = 0;
  e->all_launches = 0;
  if (rc == GD_OK) rc = configure(e, best);
  char line[160];
  snprintf(line, sizeof line, "chosen: warps=%d kpl=%d ab=%d stage=%d\n", best.warps_per_cta, best.kpl, best.ab,
           best.stage);
  rep += line;
  if (report && report_len > 0) {
    std::strncpy(report, rep.c_str(), (size_t)report_len - 1);
    report[report_len - 1] = 0;
  }
  return rc;
}

// ---------------------------------------------------- checkpoint / resume
namespace {
constexpr uint64_t kSnapMagic = 0x3130504e53444723ull;  // "#GDSNP01"

// Snapshot layout: SnapHeader, then per job a SnapJob, then per job its
// ReplicaMC[nrep], int run_acc[nrep] and RepStats[nrep], in job order.
struct SnapHeader {
  uint64_t magic;
  int32_t njob;
  int32_t step;
};
struct SnapJob {
  int32_t nrep, rid_base;
  uint32_t key0, key1;
};

size_t snap_job_bytes(const DevJob &J)
{
  return (sizeof(ReplicaMC) + sizeof(int) + sizeof(RepStats)) * (size_t)J.nrep;
}
}  // namespace

size_t gd_ensemble_snapshot_bytes(const gd_ensemble_t *e)
{
  if (!e) return 0;
  size_t b = sizeof(SnapHeader) + sizeof(SnapJob) * e->jobs.size();
  for (const auto &j : e->jobs) b += snap_job_bytes(j.dj);
  return b;
}

int gd_ensemble_snapshot(gd_ensemble_t *e, void *buf, size_t bytes)
{
  if (!e || !buf) return fail(GD_E_INVALID, "null argument");
  if (bytes < gd_ensemble_snapshot_bytes(e))
    return fail(GD_E_INVALID, "snapshot buffer of %zu bytes, %zu needed", bytes, gd_ensemble_snapshot_bytes(e));
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  GD_TRY(check_err(e));
  unsigned char *p = (unsigned char *)buf;
  SnapHeader h{kSnapMagic, (int32_t)e->jobs.size(), (int32_t)e->step};
  std::memcpy(p, &h, sizeof h);
  p += sizeof h;
  for (const auto &j : e->jobs) {
    const SnapJob sj{j.dj.nrep, j.dj.rid_base, j.dj.key0, j.dj.key1};
    std::memcpy(p, &sj, sizeof sj);
    p += sizeof sj;
  }
  for (const auto &j : e->jobs) {
    const DevJob &J = j.dj;
    GD_CUDA(cudaMemcpyAsync(p, J.rep, sizeof(ReplicaMC) * J.nrep, cudaMemcpyDeviceToHost, e->st));
    p += sizeof(ReplicaMC) * J.nrep;
    GD_CUDA(cudaMemcpyAsync(p, J.run_acc, sizeof(int) * J.nrep, cudaMemcpyDeviceToHost, e->st));
    p += sizeof(int) * J.nrep;
    GD_CUDA(cudaMemcpyAsync(p, J.stats, sizeof(RepStats) * J.nrep, cudaMemcpyDeviceToHost, e->st));
    p += sizeof(RepStats) * J.nrep;
  }
  GD_CUDA(cudaStreamSynchronize(e->st));
  return GD_OK;
}

int gd_ensemble_restore(gd_ensemble_t *e, const void *buf, size_t bytes)
{
  if (!e || !buf) return fail(GD_E_INVALID, "null argument");
  if (bytes < sizeof(SnapHeader)) return fail(GD_E_INVALID, "snapshot of %zu bytes", bytes);
  const unsigned char *p = (const unsigned char *)buf;
  SnapHeader h;
  std::memcpy(&h, p, sizeof h);
  if (h.magic != kSnapMagic) return fail(GD_E_INVALID, "not an ensemble snapshot");
  if (h.njob != (int32_t)e->jobs.size())
    return fail(GD_E_INVALID, "snapshot of %d jobs, ensemble has %zu", h.njob, e->jobs.size());
  if (bytes < gd_ensemble_snapshot_bytes(e))
    return fail(GD_E_INVALID, "snapshot of %zu bytes, this ensemble's is %zu", bytes, gd_ensemble_snapshot_bytes(e));
  if (h.step < 0) return fail(GD_E_INVALID, "snapshot step %d", h.step);
  p += sizeof h;
  for (size_t k = 0; k < e->jobs.size(); ++k) {
    SnapJob sj;
    std::memcpy(&sj, p, sizeof sj);
    p += sizeof sj;
    const DevJob &J = e->jobs[k].dj;
    // the Philox draws are keyed by (seed, replica, step): a snapshot continues
    // bit for bit only in an ensemble of the same replicas and seeds
    if (sj.nrep != J.nrep || sj.rid_base != J.rid_base || sj.key0 != J.key0 || sj.key1 != J.key1)
      return fail(GD_E_INVALID, "snapshot job %zu: replicas/seed differ from the ensemble's", k);
  }
  GD_TRY(set_device(e->device));
  GD_CUDA(cudaStreamSynchronize(e->st));
  for (const auto &j : e->jobs) {
    const DevJob &J = j.dj;
    GD_CUDA(cudaMemcpyAsync(J.rep, p, sizeof(ReplicaMC) * J.nrep, cudaMemcpyHostToDevice, e->st));
    p += sizeof(ReplicaMC) * J.nrep;
    GD_CUDA(cudaMemcpyAsync(J.run_acc, p, sizeof(int) * J.nrep, cudaMemcpyHostToDevice, e->st));
    p += sizeof(int) * J.nrep;
    GD_CUDA(cudaMemcpyAsync(J.stats, p, sizeof(RepStats) * J.nrep, cudaMemcpyHostToDevice, e->st));
    p += sizeof(RepStats) * J.nrep;
  }
  GD_CUDA(cudaStreamSynchronize(e->st));
  e->step = h.step;
  return GD_OK;
}

int gd_ensemble_destroy(gd_ensemble_t *e)
{
  destroy(e);
  return GD_OK;
}

}  // extern "C"

// ------------------------------------------------------------- layout --
// Sizes and offsets of the boundary structs, for bindings that mirror them.
extern "C" long long gd_layout(const char *what)
{
  if (!what) return -1;
  const std::string w(what);
#define GD_L(name, expr) \
  if (w == name) return (long long)(expr);
  GD_L("sizeof.Complex", sizeof(Complex))
  GD_L("sizeof.Record", sizeof(Record))
  GD_L("sizeof.ReplicaMC", sizeof(ReplicaMC))
  GD_L("sizeof.EnePara", sizeof(EnePara))
  GD_L("sizeof.EnePara0", sizeof(EnePara0))
  GD_L("sizeof.Ligand", sizeof(Ligand))
  GD_L("sizeof.Protein", sizeof(Protein))
  GD_L("sizeof.Kde", sizeof(Kde))
  GD_L("sizeof.Mcs", sizeof(Mcs))
  GD_L("sizeof.ParaT", sizeof(ParaT))
  GD_L("Complex.lig", offsetof(Complex, lig))
  GD_L("Complex.prt", offsetof(Complex, prt))
  GD_L("Complex.psp", offsetof(Complex, psp))
  GD_L("Complex.kde", offsetof(Complex, kde))
  GD_L("Complex.mcs", offsetof(Complex, mcs))
  GD_L("Complex.enepara", offsetof(Complex, enepara))
  GD_L("Complex.temp", offsetof(Complex, temp))
  GD_L("Complex.replica", offsetof(Complex, replica))
  GD_L("Complex.size", offsetof(Complex, size))
  GD_L("Complex.mcpara", offsetof(Complex, mcpara))
  GD_L("Complex.lig_file", offsetof(Complex, lig_file))
  GD_L("Complex.rep_begin", offsetof(Complex, rep_begin))
  GD_L("Complex.rep_end", offsetof(Complex, rep_end))
  GD_L("Complex.signal", offsetof(Complex, signal))
  GD_L("EnePara.w", offsetof(EnePara, w))
  GD_L("EnePara.hpl0", offsetof(EnePara, hpl0))
  GD_L("EnePara.kde2", offsetof(EnePara, kde2))
  GD_L("Record.next_entry", offsetof(Record, next_entry))
  GD_L("sizeof.gd_job_desc_t", sizeof(gd_job_desc_t))
  GD_L("sizeof.gd_pocket_desc_t", sizeof(gd_pocket_desc_t))
  GD_L("sizeof.gd_server_config_t", sizeof(gd_server_config_t))
  GD_L("sizeof.gd_request_t", sizeof(gd_request_t))
  GD_L("sizeof.gd_result_t", sizeof(gd_result_t))
  GD_L("sizeof.gd_server_stats_t", sizeof(gd_server_stats_t))
  GD_L("sizeof.gd_load_args_t", sizeof(gd_load_args_t))
  GD_L("sizeof.gd_cluster_t", sizeof(gd_cluster_t))
  GD_L("gd_server_stats_t.warps_per_cta", offsetof(gd_server_stats_t, warps_per_cta))
  GD_L("gd_result_t.t_done", offsetof(gd_result_t, t_done))
#undef GD_L
  return -1;
}

// ------------------------------------------------------ force field --
// OptimizeEnepara (src/frontend/util_optimize_soa.C:489-540): the same float
// operations in the same order, so the tables match the reference bit for bit.
extern "C" int gd_optimize_enepara(const EnePara0 *e0, EnePara *e)
{
  if (!e0 || !e) return fail(GD_E_INVALID, "null argument");
  std::memset(e, 0, sizeof(EnePara));
  const float sqrt_2_pi = sqrtf(2.0f * 3.1415926535f);
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      const float tmp = e0->vdw[j][i][0] * e0->lj[2];
      e->p1a[i][j] = 2.0f * e0->vdw[j][i][1] * powf(tmp, 9.0f);
      e->p2a[i][j] = 3.0f * e0->vdw[j][i][1] * powf(tmp, 6.0f);
    }
  e->lj0 = e0->lj[0];
  e->lj1 = e0->lj[1];
  e->el1 = e0->el[1];
  e->el0 = e0->el[0];
  e->a1 = 4.0f - 3.0f * e0->el[0];
  e->b1 = 2.0f * e0->el[0] - 3.0f;
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      e->pmf0[i][j] = e0->pmf[j][i][0];
      e->pmf1[i][j] = e0->pmf[j][i][1];
      e->hdb0[i][j] = e0->hdb[j][i][0];
      e->hdb1[i][j] = 1.0f / e0->hdb[j][i][1];
    }
  for (int i = 0; i < GD_MAXTP4; ++i) e->hpp[i] = e0->hpp[i];
  for (int i = 0; i < GD_MAXTP2; ++i) {
    e->hpl0[i] = e0->hpl[i][0];
    e->hpl1[i] = e0->hpl[i][1];
    e->hpl2[i] = logf(1.0f / (e->hpl1[i] * sqrt_2_pi));
  }
  e->kde2 = -0.5f / (e0->kde * e0->kde);
  e->kde3 = powf(e0->kde * sqrt_2_pi, 3.0f);
  for (int i = 0; i < GD_MAXWEI; ++i) {
    e->w[i] = e0->w[i];
    e->a_para[i] = e0->a_para[i];
    e->b_para[i] = e0->b_para[i];
  }
  return GD_OK;
}

// ------------------------------------------------------------ timing --
extern "C" void *gd_ensemble_stream(const gd_ensemble_t *e) { return e ? (void *)e->st : nullptr; }

namespace {
// Independent FMA chains: 8 accumulators per thread so the FMA pipe, not
// latency, bounds the loop; the result is stored so nothing is dead code.
__global__ void fma_peak_kernel(float *out, int iters, float a, float b)
{
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
        x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}
}  // namespace

// Measured FP32 FMA throughput of the current device in TFLOP/s (2 flops per FMA).
extern "C" int gd_fp32_peak(double *tflops)
{
  if (!tflops) return fail(GD_E_INVALID, "null argument");
  int dev = 0, nsm = 0;
  GD_CUDA(cudaGetDevice(&dev));
  GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 512, blocks = nsm * 4, iters = 4096;
  float *out = nullptr;
  GD_CUDA(cudaMalloc(&out, sizeof(float) * threads * blocks));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  fma_peak_kernel<<<blocks, threads>>>(out, 64, 0.999f, 1e-3f);  // warm-up
  cudaEventRecord(a);
  fma_peak_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
  cudaEventRecord(b);
  const cudaError_t e = cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  if (e != cudaSuccess) return fail(GD_E_CUDA, "gd_fp32_peak: %s", cudaGetErrorString(e));
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * threads * blocks;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return GD_OK;
}
