// gd_internal.h -- device-side layout of the docking data and kernel entry
// points shared by the translation units of libgdock.so.
//
// The reference keeps everything in one fixed-capacity 6.58 MB Complex blob
// and lets every CUDA block walk it through the read-only cache
// (src/backend_gpu/kernel_cuda_l1_montecarlo.cu:142-228).  Here the blob is
// only the boundary format: it is packed once into compact structure-of-arrays
// buffers sized to the actual problem:
//
//   pocket conformation  pos[P] float4 (x, y, z, ele), aux[P] float2 (hpp_eff,
//                        type): hydrophobic-contact points first, each part
//                        with the hydrogen-bond point types first, each group
//                        sorted by point type, padded with inert points
//   force-field tables   tab4[24][32] float4 (1/p1a, -p2a/p1a, -pmf0, pmf1) for the FP32 pair loop
//                        tab2[24][32] float2 (hdb1 c, -hdb0 hdb1 c), zero where hdb0 <= 0.1
//                        ref4[24][32] float4 (p1a, p2a, hdb0, hdb1) as in EnePara (FP64, plain)
//   ligand conformation  lig[L] float4 (x, y, z, charge), atoms grouped by type; the
//                        rotated pose of a replica lives in shared memory with
//                        every value twice (packed f32x2 operands)
//   KDE points           kde[K] float4 (x, y, z, type), sorted by type, with
//                        per-type ranges
//   MCS templates        mcs[L][M] float4 (x, y, z, valid), atom-major
//   pocket potential     psp[prt conf][24][P] pre-gathered per sorted point,
//                        pspmask[prt conf][P] its non-zero ligand types, and
//                        pcell[prt conf][] its non-zero cells for the ligand's
//                        types (the atom-pair pair loop's form)
//
// Every array a CTA stages into shared memory is a multiple of 16 bytes and
// starts 16-byte aligned, so it can be copied with one 1-D bulk (TMA) copy.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "gdock_types.h"

namespace gd {

constexpr int kLigTypes = GD_MAXTP2;     // 24 ligand atom types
constexpr int kTabCols = 32;             // point-type columns (30 used, 30 = inert padding)
constexpr int kPadType = 30;             // point type given to padding points
constexpr int kMaxAtoms = 128;           // ligand atoms per job on the batched path
constexpr int kPointAlign = 128;         // pocket conformations padded to this many points
constexpr int kMaxTemps = GD_MAX_TMP;
constexpr int kMaxCtaThreads = 512;      // launch bound of the batched kernel (<= 16 replica-warps)
// c = sqrt(log2(e) / 2): exp(-h^2/2) = 2^-(h c)^2 (scaled hydrogen-bond table entries)
constexpr double kHdbC = 0.8493218002880191;

// Force-field parameters of one job, in the order the kernels stage them.
// The FP32 pair code uses algebraically rearranged forms of the reference
// formulas whose constants are precomputed here (values in the comments).
// FP32 pair-table entry of one (ligand type, point type):
// (1/p1a, -p2a/p1a, -pmf0, pmf1).  The Lennard-Jones term
// (p1 - p2) / (p1 lj0 (1 + lj1 d^2) + 1) with p1 = p1a / d^9, p2 = p2a / d^6
// divided through by p1 is (1 - (p2a/p1a) d^3) / (lj0 + lj0 lj1 d^2 + d^9 / p1a),
// which needs p1a > 0 (true for every type pair of the reference's parameter
// file; the packers refuse others); d - pmf0 is d + (-pmf0), exactly.
// Padding point types get 1/p1a = +inf: the denominator is infinite and every
// term exactly zero.
__host__ __device__ inline float4 tab4_entry(float p1a, float p2a, float pmf0, float pmf1)
{
  return make_float4((float)(1.0 / (double)p1a), (float)(-(double)p2a / (double)p1a), -pmf0, pmf1);
}
__host__ __device__ inline float4 tab4_padding() { return make_float4(INFINITY, 0.f, 0.f, 0.f); }

// The scalar parameters come first and the per-type tables last: the FP32
// batched kernel stages only the scalar prefix in shared memory (it reads the
// tables from global memory once per work item to build its per-atom-pair
// tables); the FP64 and plain kernels stage the whole struct.
struct alignas(16) DevParams {
  uint32_t hdbmask[kLigTypes];        // bit pt set where (ligand type, point type) has hdb0 > 0.1
  float hpl0[kLigTypes], hpl1[kLigTypes], hpl2[kLigTypes];
  float a_para[12], b_para[12], w[12];
  float lj0, lj1, el0, el1, inv_el1, a1, b1, kde2, kde3_inv;
  float lj01;                         // lj0 * lj1
  float ele_a, ele_b, ele_d2max;      // a1 el1^2, b1 el1^3, 1/el1^2 (near-field branch: d^2 < 1/el1^2)
  float hdb_cinv;                     // 1/c
  float move_scale[6];
  float kde3;                         // (h sqrt(2 pi))^3: the FP64 kernels divide by it
  float pad_;
  float4 tab4[kLigTypes][kTabCols];   // 1/p1a, -p2a/p1a, -pmf0, pmf1 (tab4_entry); the point-type
                                      // padding columns (>= 30) give exactly zero for every term
  float2 tab2[kLigTypes][kTabCols];   // hdb1*c, -hdb0*hdb1*c with c = sqrt(log2(e)/2);
                                      // zero where hdb0 <= 0.1 (no hydrogen-bond parameters)
};
static_assert(sizeof(DevParams) % 16 == 0, "DevParams must be a multiple of 16 bytes");
// bytes of the scalar prefix (a multiple of 16: tab4 is 16-byte aligned)
constexpr size_t kParamScalarBytes = offsetof(DevParams, tab4);
static_assert(kParamScalarBytes % 16 == 0, "the scalar prefix is bulk-copied");

// Per-replica running statistics, accumulated on the device in FP64.
struct alignas(16) RepStats {
  double e_sum;          // sum of the accepted-state total energy, one sample per step
  double e_sum2;         // sum of squares
  double best_e;         // lowest total energy seen
  long long n_steps;     // steps taken
  long long n_accept;    // accepted moves
  long long n_exch_try;  // exchange attempts involving this replica
  long long n_exch_acc;  // accepted exchanges
  float best_mm[6];      // pose of best_e
  int best_step;
  int pad_;
};

// One docking job: one ligand (all its conformations) against one pocket.
struct DevJob {
  // ligand
  int natom;               // L
  int nlig;                // ligand conformations
  int lstride;             // float4 stride between ligand conformations (>= L)
  const float4 *lig;       // [nlig][lstride] (x, y, z, charge), type-grouped order
  const int2 *lgrp;        // [L] (atom type, end index of its type group), type-grouped order
  const float *lcenter;    // [nlig][3] ligand centre in the lab frame
  // pocket
  int npoint_pad;          // padded point count (multiple of kPointAlign)
  int nprt;                // protein conformations
  const float4 *pos;       // [nprt][npoint_pad]
  const float2 *aux;       // [nprt][npoint_pad] (hpp if cdc == 1 else 0, point type)
  const int *ncdc;         // [nprt] hydrophobic-contact (cdc == 1) points, placed first in each conformation
  const float *pcenter;    // [nprt][3] pocket centre
  const float *psp;        // [nprt][24][npoint_pad]
  const uint32_t *pspmask; // [nprt][npoint_pad] bit t set where psp[.][t][p] != 0
  // the same potential as a list of its non-zero cells (sorted point p, ligand type t) per
  // conformation, for the types the ligand has, ordered by type, then point: cell k <
  // pcell_cnt[c] of conformation c is the int4 pair pcell[2 (c * pcell_stride + k) + {0, 1}] =
  // (bits of x, y, z of point p and of the value), (beg | end << 16, bits of -pmf0 of (t, type
  // of p), t, p), [beg, end) the atoms of type t in the type-grouped ligand
  const int4 *pcell;
  const int *pcell_cnt;    // [nprt]
  int pcell_stride;        // cells per conformation
  // KDE
  int nkde;
  const float4 *kde;       // [nkde]
  int kbeg[kLigTypes];
  int kcnt[kLigTypes];
  // the same as a list of (KDE point, ligand type group) slots, one per KDE point of a type the
  // ligand has, in the grouped ligand's type order: slot s is the int4 pair kslot[2 s + {0, 1}] =
  // (bits of x, y, z of the point and of 1/(points of its type)), (beg | end << 16, 0, 0, 0),
  // [beg, end) the group's atoms; nkslot <= nkde (the atom-pair form's KDE pass)
  int nkslot;
  const int4 *kslot;
  // MCS
  int nmcs;
  const float4 *mcs;       // [L][nmcs]
  const float *tcc;        // [nmcs]
  // temperatures
  int ntmp;
  const float *minus_beta; // [ntmp]
  // parameters
  const DevParams *par;
  const float4 *ref4;      // [24][32] (p1a, p2a, hdb0, hdb1) as in EnePara, hdb zero where hdb0 <= 0.1
                           // (FP64 and plain kernels)
  // replicas (layout of the reference's replica array: index
  // n_tmp*n_lig*p + n_lig*t + l, src/frontend/util.C:380)
  int nrep;
  ReplicaMC *rep;          // [nrep]
  int *run_acc;            // [nrep] accept flag of the last step
  RepStats *stats;         // [nrep]
  Record *rec;             // [nrep] or nullptr
  uint32_t key0, key1;     // Philox key (job seed)
  int rid_base;            // global index of local replica 0 (Philox counter, exchange partners)
  int nrep_total;          // replicas of the whole ensemble (nlig * nprt * ntmp)
  // per-job scheduling state (zero for ensembles; set each round by the server)
  int step0;               // added to the launch's first step: the job's own step count
  int nsteps;              // > 0: steps this job runs in a launch (<= the launch's), else the launch's
  int xsweep;              // exchange sweep run for this job by exchange_jobs_kernel (< 0: none)
  int pad_;
};

// One unit of work of the batched kernel: `count` consecutive replicas of
// one job that share protein conformation `prt`.
struct WorkItem {
  int job;
  int prt;
  int rep0;
  int count;
};

// Kernel configuration chosen by the autotuner.
struct TileConfig {
  int warps_per_cta;   // replicas per CTA (one warp each)
  int kpl;             // pocket points per lane per row (1, 2 or 4)
  int ab;              // ligand atoms per register block (4 or 8)
  int stage = 1;       // 1: stage the protein conformation in shared memory, 0: read it through L1
  int group = 1;       // warps per replica (1, 2, 4 or 8; FP32 only): a replica's pair rows, KDE points and
                       // hydrophobic sums split over them (latency mode)
};

// Pair-tile shape where the caller leaves it to the library (option value 0):
// 4 points per lane with one warp per replica, 2 in latency mode, whose warps
// share a replica's rows (shorter rows deal out more evenly); 8-atom
// hydrophobic blocks.  Measured on the batched FP32 kernel: 4 x 8 runs the
// 3520-replica Dock call 1.8 % and a one-replica 600-point complex 10 %
// faster than 2 x 8, and 4 points per lane make a replica on 4 or 8 warps
// 14-25 % slower.
inline void default_pair_tile(int group, int &kpl, int &ab)
{
  if (kpl == 0) kpl = group > 1 ? 2 : 4;
  if (ab == 0) ab = 8;
}

enum Precision { kFP32 = 0, kFP32Kahan = 1, kFP64 = 2 };

// Launch flags of the Monte Carlo kernels.
enum McFlags {
  kMcRecord = 1,         // append accepted states to Record
  kMcResetRecord = 2,    // this launch starts a dump chunk (next_entry = 0)
  kMcStoreAccept = 4,    // write the running accept flag into ReplicaMC.is_accept at the end
  kMcInitial = 8,        // initial-energy evaluation: no move, forced accept
};

// Error flags written by kernels into a device word.
enum DevError { kErrNone = 0, kErrTimeout = 1, kErrSize = 2, kErrPack = 4 };

// ---- kernels (gd_mc.cu) ----------------------------------------------------

// Arguments of the batched kernel (Monte Carlo mode and pose-evaluation mode).
struct KArgs {
  const DevJob *jobs;
  const WorkItem *items;
  int n_items;
  int *queue;
  int *err;
  int s_begin, nsteps, flags;
  const int *d_step;       // if set, steps start at *d_step + s_begin (graph replay)
  int P, Kst, lig_slots;   // smem layout (maxima over the launched jobs); P = 0: pocket read from global memory
  uint32_t wait_limit;     // microseconds a bounded shared-memory wait lasts before it gives up (0: one second)
  uint16_t stall_bytes;    // test hook: bytes announced to the staging barrier that no copy delivers, so
                           // that its bounded wait runs out (0 in normal use)
  uint16_t group;          // warps per replica (TileConfig::group); 0 reads as 1.  Two 16-bit fields in the
                           // place of one 32-bit one: the size of this struct changes the kernels' register
                           // allocation (measured), so it is kept
  // pose evaluation
  const int *conf;
  const float *mm;
  float *out;
  double *out64;
  float *raw;
};

// Shared-memory bytes of the batched kernel for pocket conformations of P
// points, Kst KDE points staged, lig_slots ligand atoms and `warps` replicas per CTA.
size_t kernel_smem_bytes(int P, int Kst, int lig_slots, int warps, int precision, int group = 1);

// Resident CTAs per SM of the batched kernel for this configuration (0 if it cannot launch).
int kernel_occupancy(int mode, int precision, const TileConfig &tc, size_t smem);

// mode 0: Monte Carlo chunk over the work items; mode 1: pose evaluation.
cudaError_t launch_kernel(int mode, int precision, const TileConfig &tc, const KArgs &a, int grid, cudaStream_t st);

// Pose evaluation reading the packed job from global memory (8 poses per 256-thread CTA, grid-stride).
cudaError_t launch_eval_global(int precision, const DevJob *d_job, const int *conf, const float *mm, int n,
                               float *out, float *raw, int *err, int grid, cudaStream_t st);

// Replica-exchange sweep over all jobs (d_xoff: [2][njob+1] pair-count prefix sums per
// parity; total: the larger of the two totals).  With d_step, the sweep index is
// (*d_step + chunk) / spx - 1, else x.
cudaError_t launch_exchange_all(const DevJob *d_jobs, const int *d_xoff, int njob, int total, int x,
                                const int *d_step, int spx, int chunk, cudaStream_t st);
// *d_step += n on the stream.
cudaError_t launch_set_step(int *d_step, int v, cudaStream_t st);
// One exchange sweep per job, sweep index jobs[j].xsweep (skipped when < 0);
// max_pairs bounds groups x pairs over the jobs.
cudaError_t launch_exchange_jobs(const DevJob *d_jobs, int njob, int max_pairs, cudaStream_t st);
cudaError_t launch_advance_step(int *d_step, int n, cudaStream_t st);

// Replica-exchange sweep x of one job (ngroup = nprt * nlig groups of ntmp temperatures).
cudaError_t launch_exchange(const DevJob *d_job, int ngroup, int ntmp, int x, cudaStream_t st);

// The plain kernel (gd_plain.cu): one CTA per replica, the reference's launch structure.
cudaError_t launch_plain(const DevJob *d_job, int nrep, int s_begin, int nsteps, int flags, int *d_err,
                         cudaStream_t st);

}  // namespace gd
