// gd_pack.h -- host-side job description and packing into the device layout.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "gd_internal.h"
#include "gdock.h"

namespace gd {

// Phase timing on stderr when the environment variable GDOCK_TRACE is set:
// host wall-clock milliseconds since the previous mark of the same tracer.
struct Tracer {
  explicit Tracer(const char *scope);
  void mark(const char *phase);
  bool on;
  const char *scope;
  double t_last;
};

// Sets the calling thread's error message; returns `code`.
int fail(int code, const char *fmt, ...);

// Test hook (option "fail_alloc"): the next n device allocations of job
// packing report GD_E_NOMEM as a failed cudaMalloc would, without calling it.
void set_injected_alloc_failures(int n);
int injected_alloc_failures();
// True (and one fewer left) if the next allocation is to fail.
bool take_injected_alloc_failure();

#define GD_CUDA(call)                                                                                \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return ::gd::fail(GD_E_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#define GD_TRY(expr)             \
  do {                           \
    const int rc_ = (expr);      \
    if (rc_ != GD_OK) return rc_; \
  } while (0)

// Pocket (protein conformations) in dense host arrays.
struct PocketData {
  int nconf = 0, P = 0;              // P = max points over conformations
  std::vector<int> npts;             // [nconf]
  std::vector<float> xyz;            // [nconf][P][3]
  std::vector<int> type, cls, cdc, seq3r;  // [nconf][P]
  std::vector<float> hpp, ele;       // [nconf][P]
  std::vector<float> center;         // [nconf][3]
  uint32_t hdb_types = 0;            // point types with a hydrogen-bond parameter (sorted first in each part)
};

// Point types with a hydrogen-bond parameter for some ligand type (hdb0 > 0.1,
// the reference's guard): bit pt.
uint32_t hdb_point_types(const EnePara &ep);

// One docking job in dense host arrays.
struct JobData {
  int L = 0, nlig = 0;
  std::vector<float> lxyz;           // [nlig][L][3], ligand-centre frame, input atom order
  std::vector<int> ltype;            // [L]
  std::vector<float> lcharge;        // [L]
  std::vector<float> lcenter;        // [nlig][3]
  int K = 0;
  std::vector<float> kxyz;           // [K][3]
  std::vector<int> ktype;            // [K]
  int M = 0;
  std::vector<float> mxyz;           // [M][L][3]
  std::vector<float> tcc;            // [M]
  int psp_ncol = 0;
  std::vector<float> psp;            // [24][psp_ncol]
  int ntmp = 0;
  std::vector<float> minus_beta;     // [ntmp]
  float move_scale[6] = {0, 0, 0, 0, 0, 0};
  uint64_t seed = 0;
  int nprt = 0;                      // protein conformations of the pocket
  bool cell_room = false;            // pocket-specific cells: room for any potential of these shapes
  std::vector<ReplicaMC> reps;       // replicas to run (a contiguous range)
  int rid_base = 0;                  // ensemble index of reps[0]
  int nrep_total = 0;                // nlig * nprt * ntmp
};

// Device copy of a pocket: type-sorted, padded conformations.
struct DevPocket {
  int nconf = 0, Ppad = 0;
  float4 *pos = nullptr;             // [nconf][Ppad]
  float2 *aux = nullptr;             // [nconf][Ppad]
  float *center = nullptr;           // [nconf][3]
  int *ncdc = nullptr;               // [nconf] hydrophobic-contact points (placed first)
  std::vector<int> scls, sseq;       // host: class and residue serial of each sorted point
  std::vector<float4> spos;          // host: pos of each sorted point
  std::vector<int> stype;            // host: point type of each sorted point (kPadType for padding)
  uint32_t hdb_types = 0;            // the PocketData::hdb_types it was sorted with
  void *arena = nullptr;
  size_t bytes = 0;
};

// Device copy of a job.
struct DevJobBuf {
  DevJob dj{};                       // device pointers (host copy of the struct)
  void *arena = nullptr;
  size_t bytes = 0;
  bool own_rec = false;
  int pocket = 0;
};

int pocket_from_complex(const Complex *c, PocketData &pk);
int job_from_complex(const Complex *c, int rep_begin, int rep_end, uint64_t seed, JobData &jd);
int pocket_from_desc(const gd_pocket_desc_t &d, PocketData &pk);
int job_from_desc(const gd_job_desc_t &d, int nprt, JobData &jd);

// Replica layout of SetReplica (src/frontend/util.C:371-406).
void default_replicas(int nlig, int nprt, int ntmp, std::vector<ReplicaMC> &out);

int build_params(const EnePara &ep, const float move_scale[6], DevParams &p);

// reuse: a previous packing whose device arena is taken over (and refilled
// with copies on `st`) when it has exactly the size the new packing needs;
// otherwise a new arena is allocated and `reuse` is left to the caller.
int pack_pocket(const PocketData &pk, DevPocket &out, const DevPocket *reuse = nullptr, cudaStream_t st = nullptr);
// rec: external device Record array (nullptr with want_records allocates one).
int pack_job(const JobData &jd, const DevPocket &pk, const EnePara &ep, bool want_records, Record *rec,
             DevJobBuf &out, const DevJobBuf *reuse = nullptr, cudaStream_t st = nullptr);
// Stream-ordered variant (cudaMallocAsync + a copy on `st`), no records.
int pack_job_async(const JobData &jd, const DevPocket &pk, const EnePara &ep, cudaStream_t st, DevJobBuf &out);
// Best poses of a job's replicas, their RMSD to a reference pose and their
// leader clustering in energy order (gd_analysis.cu).
int cluster_job(const DevJob &J, const DevJob *d_job, cudaStream_t st, int ref_lig, const float ref_mm[6],
                float rmsd_cut, gd_cluster_t *clusters, int max_clusters, int *n_clusters, int *cluster_of,
                float *rmsd_to_ref);
// Destination of the device-side packer (gd_devpack.cu): device arrays laid
// out as the host packer lays them out, and the DevJob header to write.
// err[4]: flag (kErrPack), failure kind, field id, value (zeroed by the
// caller).  Expectations (-1 or 0: none) bound what the packer may write:
// a Complex of other shapes fails with kPackFailShape and writes nothing past
// the validation.
struct PackDst {
  DevJob *job;
  DevParams *par;
  float4 *ref4;
  int *err;
  int2 *lgrp;
  float *lcenter, *pcenter, *tcc;
  float4 *lig, *kde, *mcs;
  float4 *pos;
  float2 *aux;
  int *ncdc;
  float *psp;
  uint32_t *pspmask;
  int4 *pcell;         // pocket-specific cells (nullptr: none; only the per-type-group form reads the job)
  int4 *kslot;         // KDE slots, kde_cap of them (nullptr: none, as pcell)
  int *pcell_cnt;
  int pcell_stride;    // cells per conformation the array holds
  int kde_cap;         // KDE points the kde array holds
  int Ppad;            // > 0: padded points per conformation the arrays hold (else from the Complex)
  int nkde_expect;     // >= 0: KDE points of ligand types the arrays hold
  int expect_L, expect_nlig, expect_nprt, expect_M, expect_ntmp;  // >= 0: the shapes the arrays hold
  // replicas (null rep: none): the Complex's replicas [rep_begin, rep_begin + nrep)
  ReplicaMC *rep;
  int *run_acc;
  RepStats *stats;
  float *minus_beta;
  Record *rec;
  int rep_begin, nrep, nrep_total;
  uint32_t key0, key1;
};
enum { kPackFailCapacity = 1, kPackFailInput = 2, kPackFailShape = 3 };
enum { kFieldNLig = 1, kFieldNPrt, kFieldNatom, kFieldNatomConf, kFieldNpoint, kFieldKde, kFieldMcs, kFieldLigType,
       kFieldPrtType, kFieldSeq3r, kFieldMcsRow, kFieldP1a, kFieldNTmp, kFieldReplica, kFieldPcell };
// Launches the packer on `st` (setup, pocket, ligand kernels); failures stay in D.err.
cudaError_t device_pack(const Complex *d_cx, const PackDst &D, cudaStream_t st);
const char *pack_field_name(int field);

void free_pocket(DevPocket &p);
void free_job(DevJobBuf &j);
void free_job_async(DevJobBuf &j, cudaStream_t st);

}  // namespace gd
