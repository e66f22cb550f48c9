/*
 * gdock.h -- C ABI of libgdock.so, the B200 (sm_100a) Monte Carlo docking
 * backend.
 *
 * Part 1 is the drop-in boundary: the functions a GeauxDock frontend calls
 * around its GPU backend, with the reference's names and argument shapes.
 * Two deliberate changes from the reference signatures:
 *   - every function returns int (GD_OK = 0, negative GD_E_* on failure;
 *     gd_last_error() gives the message) where the reference prints and
 *     calls exit() (src/module/yeah/cuda/runtime/wrapper.h:21-64);
 *   - curandState** becomes gd_rng_t**, an opaque counter-based Philox
 *     handle (seeded, reproducible) in place of time-seeded XORWOW states
 *     (src/backend_gpu/backend_gpu.cu:49-59).
 * The array arguments (Complex **cd, Record **rd, ParaT **pt, gd_rng_t **rng)
 * have one entry per GPU, as the reference's cd[NGPU] arrays
 * (src/main_gpu/geauxdock.C:296-302); the GPU count is gd_set_ngpu()
 * (default 1, or the GDOCK_NGPU environment variable).
 *
 * Part 2 is additive: pose evaluation, resident batched ensembles, and the
 * serving loop.  All sizes are plain ints, all data plain pointers.
 */
#ifndef GDOCK_H
#define GDOCK_H

#include <stddef.h>
#include <stdint.h>

#include "gdock_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define GD_OK 0
#define GD_E_INVALID (-1)   /* malformed input (types, sizes, indices)           */
#define GD_E_NOMEM (-2)     /* device or host allocation failed                  */
#define GD_E_CAPACITY (-3)  /* input exceeds a capacity limit                    */
#define GD_E_CUDA (-4)      /* CUDA runtime error                                */
#define GD_E_TIMEOUT (-5)   /* a bounded device wait gave up                     */
#define GD_E_NODEVICE (-6)  /* no usable GPU                                     */
#define GD_E_STATE (-7)     /* call out of order (e.g. Dock before DeviceAlloc)  */
#define GD_E_BUSY (-8)      /* serving loop: admission refused (budget, queue)   */
#define GD_E_CANCELLED (-9) /* serving loop: request cancelled                   */

/* Message of the last failure on the calling thread. */
const char *gd_last_error(void);

/* Number of GPUs the reference-boundary functions spread replicas over. */
int gd_set_ngpu(int n);
int gd_get_ngpu(void);

/* ================================================ Part 1: drop-in boundary */

typedef struct gd_rng gd_rng_t;

/* src/backend_gpu/prepair.h:4 -- select the devices (prefers shared memory). */
int SetDevice(void);
/* src/backend_gpu/prepair.h:5 -- per GPU: device Complex, Record[GD_MAX_REP], RNG handle. */
int DeviceAlloc(Complex **cd, Record **rd, gd_rng_t **rng);
/* src/backend_gpu/prepair.h:6 */
int DeviceFree(Complex **cd, Record **rd, gd_rng_t **rng);
/* src/backend_gpu/prepair.h:7 -- contiguous replica range per GPU (prepair.C:64-115);
 * with replica exchange on, ranges are cut at protein-conformation boundaries. */
int SetParaT(Complex *ch, ParaT **pt);
/* src/backend_gpu/prepair.h:8 -- ch->rep_begin/rep_end set per GPU, Complex copied. */
int CopyH2D(Complex *ch, Complex **cd, ParaT **pt);
/* src/backend_gpu/backend_gpu.h:4 -- seed the Philox handles (time-seeded like the
 * reference unless gd_rng_seed() or GDOCK_SEED fixed the seed). */
int InitCurand(gd_rng_t **rng);
/* Fix the seed of one handle (reproducible runs); resets its call counter. */
int gd_rng_seed(gd_rng_t *rng, uint64_t seed);
/* Dock calls made with this handle and how many of them refilled the device
 * state kept from the previous call (same shapes and options) instead of
 * rebuilding it.  No counterpart in the reference (it allocates once in
 * DeviceAlloc and re-copies the whole Complex per call). */
int gd_rng_dock_reuse(const gd_rng_t *rng, uint64_t *calls, uint64_t *reused);
/* src/backend_gpu/backend_gpu.h:6-11 -- initial energy (forced accept), then
 * steps_total MC steps in chunks of steps_per_dump; after each chunk the
 * replicas' Record entries are copied to rh[rep_begin..rep_end].  Final
 * replica states are left in cd[g]->replica[] and also copied to
 * ch->replica[].  mcpara.steps_per_exchange > 0 adds a replica-exchange sweep
 * every that many steps (new; the reference parses but never runs it). */
int Dock(Complex *ch, Record *rh, Complex **cd, Record **rd, ParaT **pt, gd_rng_t **rng);

/* ============================================================ Part 2: additive */

/* Kernel and precision used by Dock and the ensembles. */
#define GD_KERNEL_BATCHED 0   /* one warp per replica, persistent, staged pocket */
#define GD_KERNEL_PLAIN 1     /* one CTA per replica, the reference's structure   */
#define GD_PREC_FP32 0        /* FP32 pair energies, plain reductions             */
#define GD_PREC_FP32_KAHAN 1  /* FP32 pair energies, compensated reductions       */
#define GD_PREC_FP64 2        /* FP64 pair energies                               */

/* Options: "kernel" (GD_KERNEL_*), "precision" (GD_PREC_*, default
 * GD_PREC_FP32_KAHAN), "warps" (replicas
 * per CTA, 0 = autotune), "kpl", "ab" (pair-tile shape: pocket points per
 * lane 1, 2 or 4, atoms per hydrophobic block 4 or 8; default 0, the
 * library's choice: 4, 8 with one warp per replica, 2, 8 in latency mode),
 * "graph" (1: replay whole exchange intervals from a captured CUDA graph,
 * 0: launch them one by one), "stage" (1: stage each protein conformation in
 * shared memory, 0: read it through L1, -1: choose by occupancy; pockets too
 * large to stage are always read through L1), "dock_cache" (1: Dock keeps
 * its packed device state per GPU handle and refills it in place when the next
 * Complex has the same shapes, keeping the packed protein when its bytes are
 * unchanged; 0: everything is rebuilt and freed per call), "dock_device_pack"
 * (1: that refill packs the Complex CopyH2D put on the GPU, on the GPU; 0: the
 * host re-packs it), "dock_record_direct" (1: when Dock's Record array rh is
 * page-locked host memory the GPU can address -- cudaHostAlloc, or
 * cudaHostRegister with mapping -- the kernels write each Record entry into it
 * as the chunk runs and no copy follows; entries at and past a Record's
 * next_entry keep what rh held; 0, or pageable rh: the Records go to rd[g] and
 * the whole array is copied to rh after each chunk), "device_base" (the
 * drop-in API's GPU g is CUDA device device_base + g, for one process per GPU;
 * set it before SetDevice/DeviceAlloc and keep it), "wait_limit"
 * (microseconds, on the GPU's global timer, that the kernel's bounded
 * shared-memory waits last before they give up and report GD_E_TIMEOUT;
 * 0: one second), "stall_test" (test hook, 0 in normal
 * use: ensembles announce bytes to their staging barriers that no copy
 * delivers, so that the bounded waits run out), "fail_alloc" (test hook, 0 in
 * normal use: the next n device allocations for packing a job report
 * GD_E_NOMEM without calling cudaMalloc).  Applies to objects created
 * afterwards on the calling process. */
int gd_set_option(const char *name, long long value);
long long gd_get_option(const char *name);

/* Energies of n poses of Complex c: pose i is ligand conformation conf[2i],
 * protein conformation conf[2i+1], movematrix mm[6i..6i+5].  out[10i..]:
 * the ten ReplicaMC.energy terms; raw[9i..] (may be NULL): the terms before
 * the per-atom division and normalisation; out64 (may be NULL): FP64 copy of
 * out (exact only with GD_PREC_FP64).  Host buffers; runs on GPU 0. */
int gd_eval_poses(const Complex *c, int n, const int *conf, const float *mm, int precision, float *out,
                  double *out64, float *raw);

/* Pose energies without any memory allocation.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc/cudaFree around a
 * docking call: a process whose device memory belongs to another allocator
 * (a framework's caching allocator, a pool reserved at start-up), or a
 * latency-bound serving loop that cannot afford cudaFree's device-wide
 * synchronisation.  Same result as gd_eval_poses, but every pointer is device
 * memory the caller owns: d_complex is a reference-layout Complex (for
 * example cd[g] after CopyH2D), d_conf[n][2] / d_mm[n][6] the poses,
 * d_out[n][10] and d_raw[n][9] (may be NULL) the energies; stream is a
 * cudaStream_t of the calling thread's current device (NULL: its legacy
 * default stream; a stream of another device is refused with GD_E_INVALID).
 * The call is synchronous: it ends by copying a status word back and waiting
 * for the stream, so it returns after its work on that stream finished.  The
 * packed device layout goes into one fixed scratch array in the library
 * (gd_noalloc_scratch_bytes(): 5.60 MiB, held on every GPU that loads the
 * library until exit), sized for the reference Complex's caps: larger sizes
 * fail with GD_E_CAPACITY.  The first call on a device looks up the scratch
 * array's address (set-up); make that first call before any stream capture.
 * All calls on a device share the scratch array, which keeps the last call's
 * contents: calls whose GPU work overlaps race on it. */
int gd_eval_poses_noalloc(const Complex *d_complex, int n, const int *d_conf, const float *d_mm, int precision,
                          float *d_out, float *d_raw, void *stream);
size_t gd_noalloc_scratch_bytes(void);

/* OptimizeEnepara (src/frontend/util_optimize_soa.C:489-540): raw parameters
 * -> the precomputed tables of EnePara, bit-identical to the reference. */
int gd_optimize_enepara(const EnePara0 *in, EnePara *out);

/* Cap-free description of one docking job (ligand sizes above GD_MAXLIG and
 * pockets above GD_MAXPRO are allowed).  Arrays are dense, C order. */
typedef struct gd_job_desc {
  int natom, nlig;            /* ligand atoms, ligand conformations           */
  const float *lig_xyz;       /* [nlig][natom][3] in the ligand-centre frame  */
  const int *lig_type;        /* [natom] 0..23                                */
  const float *lig_charge;    /* [natom]                                      */
  const float *lig_center;    /* [nlig][3] lab frame                          */
  int pocket;                 /* index of a pocket from gd_pocket_desc_t list */
  int nkde;
  const float *kde_xyz;       /* [nkde][3]                                    */
  const int *kde_type;        /* [nkde]                                       */
  int nmcs;
  const float *mcs_xyz;       /* [nmcs][natom][3], GD_MCS_INVALID_COORD = unset */
  const float *mcs_tcc;       /* [nmcs]                                       */
  int psp_ncol;               /* columns of psp (residue serial numbers)      */
  const float *psp;           /* [24][psp_ncol] pocket-specific potential     */
  int ntmp;
  const float *temperature;   /* [ntmp] temperatures T (minus_beta = -1/T)    */
  float move_scale[6];
  uint64_t seed;
} gd_job_desc_t;

typedef struct gd_pocket_desc {
  int npoint, nconf;
  const float *xyz;           /* [nconf][npoint][3]                           */
  const int *type;            /* [npoint] point type 0..29                    */
  const int *cls;             /* [npoint] point class c (0..3)                */
  const int *cdc;             /* [npoint] hydrophobic-contact flag            */
  const int *seq3r;           /* [npoint] residue serial number (psp column)  */
  const float *hpp;           /* [npoint]                                     */
  const float *ele;           /* [npoint]                                     */
  const float *center;        /* [nconf][3] pocket centre                     */
} gd_pocket_desc_t;

/* A resident ensemble: many jobs, their pockets, replica states and FP64
 * statistics kept in device memory and advanced by one persistent launch
 * per chunk (captured in a CUDA graph).  Replica r of job j is ligand conf
 * l, protein conf p, temperature t with r = ntmp*nlig*p + nlig*t + l. */
typedef struct gd_ensemble gd_ensemble_t;

int gd_ensemble_create(const gd_pocket_desc_t *pockets, int npocket, const gd_job_desc_t *jobs, int njob,
                       const EnePara *enepara, int device, gd_ensemble_t **out);
/* The same from reference-layout Complexes (one job each; identical proteins share a pocket). */
int gd_ensemble_create_complex(const Complex *const *cx, int n, const uint64_t *seeds, int device,
                               gd_ensemble_t **out);
/* One process per GPU: replica range [*rep_begin, *rep_end] of GPU g of ngpu
 * under SetParaT's split (exchange-aligned when exchange is on), and an
 * ensemble of just that range of a Complex.  Philox counters use the global
 * replica index, so with one seed on every GPU each replica's trajectory is
 * the same whatever the number of GPUs.  No counterpart in the reference
 * (its Dock drives every GPU from one process). */
int gd_replica_range(const Complex *ch, int ngpu, int g, int *rep_begin, int *rep_end);
int gd_ensemble_create_complex_range(const Complex *cx, int rep_begin, int rep_end, uint64_t seed, int device,
                                     gd_ensemble_t **out);
/* Initial energies (no move, forced accept). */
int gd_ensemble_init(gd_ensemble_t *e);
/* Advance every replica by nsteps MC steps, with a replica-exchange sweep
 * every steps_per_exchange steps (0 = none).  Asynchronous.  Whole exchange
 * intervals are replayed from one captured CUDA graph (Monte Carlo chunk,
 * exchange sweep, step counter). */
int gd_ensemble_run(gd_ensemble_t *e, int nsteps, int steps_per_exchange);
/* Wait for the device; kernel_ms: device time of the Monte Carlo launches
 * since the last call (CUDA events on the ensemble's stream; a replayed
 * exchange interval counts as one launch), launches: their count,
 * all_launches: every kernel of the library launched on the stream. */
int gd_ensemble_sync(gd_ensemble_t *e, double *kernel_ms, int *launches, int *all_launches);
int gd_ensemble_num_replicas(const gd_ensemble_t *e, int job);
int gd_ensemble_replicas(gd_ensemble_t *e, int job, ReplicaMC *out);
/* Per replica: {n_steps, n_accept, n_exch_try, n_exch_acc, mean E, var E, best E, best step}. */
int gd_ensemble_stats(gd_ensemble_t *e, int job, double *out8);
/* Energies of n arbitrary poses of job `job` (pose i: ligand conformation
 * conf[2i], protein conformation conf[2i+1], movematrix mm[6i..6i+5]) with the
 * resident pocket and job, in any precision; as gd_eval_poses for jobs beyond
 * the Complex caps.  Waits for the ensemble's stream first. */
int gd_ensemble_eval_poses(gd_ensemble_t *e, int job, int n, const int *conf, const float *mm, int precision,
                           float *out, double *out64, float *raw);
/* Post-analysis of job `job`: each replica's best pose (the lowest total
 * energy it visited, from its FP64 statistics), the pose's RMSD to a
 * reference pose (ligand conformation ref_lig at movematrix ref_mm; NULL: the
 * native pose, conformation 0 at zero), and the best poses clustered in
 * order of energy: a pose joins the first cluster whose lowest-energy pose is
 * within rmsd_cut (A), else it starts one.  Up to max_clusters summaries go
 * to `clusters` (all are counted in *n_clusters); cluster_of[nrep] and
 * rmsd_to_ref[nrep] (may be NULL) per replica.  No counterpart in the
 * reference (src/analysis/record.h:50-59 sketches the medoid summary). */
typedef struct gd_cluster {
  int representative;   /* replica whose best pose has the lowest energy in the cluster */
  int size;             /* best poses in the cluster */
  float relative_size;  /* size / replicas */
  float z_score;        /* (representative energy - mean best energy) / standard deviation */
  float rep_energy;     /* total energy of the representative */
  float mean_energy;    /* mean total energy of the members */
  float rep_rmsd;       /* RMSD of the representative to the reference pose, A */
  int pad_;
} gd_cluster_t;
/* Each replica's best pose: movematrix [nrep][6] and total energy [nrep] (FP64). */
int gd_ensemble_best_poses(gd_ensemble_t *e, int job, float *best_mm, double *best_energy);
int gd_ensemble_cluster(gd_ensemble_t *e, int job, int ref_lig, const float *ref_mm, float rmsd_cut,
                        gd_cluster_t *clusters, int max_clusters, int *n_clusters, int *cluster_of,
                        float *rmsd_to_ref);
/* Choose the tile shape (replicas per CTA, pair tile, pocket staging) by timing
 * candidates on a snapshot of the state (restored after each).  steps: MC
 * steps per launch to tune for (the chunk the caller runs, e.g. its exchange
 * interval); each candidate runs them on a strided sample of about two waves
 * of work items. */
int gd_ensemble_autotune(gd_ensemble_t *e, int steps, char *report, int report_len);
int gd_ensemble_destroy(gd_ensemble_t *e);
/* Checkpoint and resume of a resident ensemble: every replica's ReplicaMC,
 * its running accept flag and FP64 statistics, and the ensemble's step
 * counter, in one host buffer of gd_ensemble_snapshot_bytes() bytes.  The
 * Monte Carlo and exchange draws are keyed by (seed, replica, step), so an
 * ensemble of the same jobs and seeds restored from a snapshot continues bit
 * for bit as the uninterrupted run would.  Restore refuses a snapshot of
 * other replicas or seeds (GD_E_INVALID).  Both wait for the ensemble's
 * stream.  No counterpart in the reference: it keeps the resumable state in
 * ReplicaMC (src/common/geauxdock.h:323-336) but never saves it. */
size_t gd_ensemble_snapshot_bytes(const gd_ensemble_t *e);
int gd_ensemble_snapshot(gd_ensemble_t *e, void *buf, size_t bytes);
int gd_ensemble_restore(gd_ensemble_t *e, const void *buf, size_t bytes);
/* The CUDA stream (cudaStream_t) the ensemble launches on, for event timing. */
void *gd_ensemble_stream(const gd_ensemble_t *e);

/* ------------------------------------------------------------------ serving
 * No counterpart in the reference (it runs one Complex per Dock call).  A
 * server keeps pockets resident on one GPU and runs docking requests of any
 * ligand size against them: requests queue, are admitted while the HBM
 * budget, the replica cap and the job slots allow, and then share rounds (one
 * persistent Monte Carlo launch over every admitted job, one exchange launch)
 * with whatever else is running; finished requests leave between rounds and
 * free their memory for the queue.  A request's result does not depend on
 * the other requests (own seed, own step counter). */
typedef struct gd_server gd_server_t;

typedef struct gd_server_config {
  unsigned long long hbm_budget_bytes; /* device bytes of admitted jobs (default 100 GB) */
  int max_active_replicas;  /* replicas in one round (0: four waves of resident replica-warps) */
  int max_jobs;             /* admitted jobs at a time (result staging slots), default 256 */
  int max_replicas_per_job; /* default 1024 */
  int max_atoms;            /* largest ligand accepted (sizes the per-warp buffers), default 128 */
  int steps_per_round;      /* MC steps between scheduling decisions, default 50 */
  int kde_stage;            /* KDE points staged in shared memory (more: read through L1), default 0 */
  int warps;                /* warps per CTA, 0: occupancy model */
  int device;
  int replica_warps;        /* warps per replica, 1 (default), 2, 4 or 8: latency mode, every
                               replica's pair rows and KDE points split over that many warps;
                               -2, -4 or -8: adaptive, each round on the most warps per replica
                               (that many, or a power of two below it) for which one wave of
                               the grid holds its active replicas, else one warp per replica (a
                               request's results then depend on the load it met, within the
                               parity tolerance either way) */
} gd_server_config_t;

typedef struct gd_request {
  const gd_job_desc_t *job;   /* job->pocket indexes the server's pockets   */
  int steps;                  /* MC steps after the initial evaluation      */
  int steps_per_exchange;     /* 0: no replica exchange                     */
  ReplicaMC *replicas_out;    /* [nrep] final replica states, or NULL       */
  double *stats_out;          /* [nrep][8] as gd_ensemble_stats, or NULL    */
} gd_request_t;

typedef struct gd_result {
  long long ticket;
  int status;                 /* GD_OK, or why the request failed           */
  int nrep, steps, pad_;
  double t_submit, t_admit, t_done; /* seconds on the server's clock        */
} gd_result_t;

typedef struct gd_server_stats {
  long long submitted, completed, failed, queued, outstanding;
  long long rounds, launches;       /* rounds run, kernels launched         */
  double pose_evals;                /* replica-steps run (initial included) */
  double device_ms;                 /* device time of the rounds            */
  double now;                       /* the server's clock, seconds          */
  unsigned long long used_bytes, peak_bytes;
  int warps_per_cta, grid, max_active_replicas;
  int pocket_staged;                /* 1: pockets staged in shared memory, 0: read through L1 */
  long long latency_rounds;         /* rounds run in latency mode           */
} gd_server_stats_t;

void gd_server_config_default(gd_server_config_t *cfg);
/* Pockets are packed once and stay resident until gd_server_destroy. */
int gd_server_create(const gd_pocket_desc_t *pockets, int npocket, const EnePara *enepara,
                     const gd_server_config_t *cfg, gd_server_t **out);
/* Validates and queues a request (the job is copied; its output buffers must
 * stay valid until its result is polled).  Thread-safe. */
int gd_server_submit(gd_server_t *s, const gd_request_t *req, long long *ticket);
/* Up to max finished requests; waits up to timeout_ms (-1: until one is
 * ready or nothing is outstanding).  Returns the count (>= 0). */
int gd_server_poll(gd_server_t *s, gd_result_t *out, int max, int timeout_ms);
/* Cancels a request: a queued one is reported at once, an admitted one at
 * the next round boundary (its device memory freed stream-ordered behind the
 * rounds that still use it), with status GD_E_CANCELLED.  A request whose
 * last round is already on the GPU finishes normally instead.  GD_E_STATE if
 * its result was already reported, GD_E_INVALID for a ticket never issued.
 * Thread-safe. */
int gd_server_cancel(gd_server_t *s, long long ticket);
/* Waits until every submitted request finished (-1: no limit). */
int gd_server_drain(gd_server_t *s, int timeout_ms);
int gd_server_get_stats(gd_server_t *s, gd_server_stats_t *out);
/* Stops the loop; requests not finished yet are cancelled. */
int gd_server_destroy(gd_server_t *s);

/* ---------------------------------------------------------------- loaders
 * The reference frontend's input path for one job (src/frontend/load.C
 * loadLigand / loadLHM / loadProtein, util_optimize_soa.C Optimize*, util.C
 * SetPocketCenter / SetTemperature / SetReplica): ligand .sdf with its
 * conformer ensemble (conformers within 0.1 A RMSD of the native pose after
 * superposition dropped), the .ff file's KDE points, pocket-specific
 * potential and MCS rows of `ligand_id`, and the protein .pdb's
 * ENDMDL-terminated models, into a Complex laid out as the GPU frontend
 * builds it.  The force field comes from the caller (parameter files parsed
 * elsewhere; gd_optimize_enepara for the tables).  Returns n_rep or a
 * negative status. */
typedef struct gd_load_args {
  const char *lig_sdf, *lhm_ff, *prt_pdb;
  const char *ligand_id;        /* MCS rows of this ligand in the .ff file */
  const char *molid;            /* SDF data tag naming the molecule ("MOLID") */
  const EnePara0 *enepara0;     /* raw parameters (point ele/hpp tables) */
  const EnePara *enepara;       /* precomputed tables copied into the Complex */
  int num_temp;
  float floor_temp, ceiling_temp;
  float translation_step, rotation_step;
  int steps_total, steps_per_dump, steps_per_exchange;
} gd_load_args_t;
int gd_load_complex(const gd_load_args_t *args, Complex *out);

/* Bounds checking.  libgdock_check.so is this library with its Monte Carlo /
 * pose kernels built with -DGD_CHECK: every instrumented shared- and global-
 * memory index is compared with its array's length, and the first one out of
 * range is recorded (and redirected to element 0, so that the run completes
 * without a fault).  out4 = {1 if a violation was recorded, its site, the
 * index, the length}; reset != 0 clears the record.  Waits for the current
 * device.  In libgdock.so it returns GD_E_STATE.  No counterpart in the
 * reference (its IS_ASSERT toggle, src/common/toggle.h:21, is never used). */
int gd_check_report(int *out4, int reset);

/* Measured FP32 FMA throughput of the current GPU (TFLOP/s, 2 flops per FMA):
 * the denominator of the pair kernel's roofline. */
int gd_fp32_peak(double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* GDOCK_H */
