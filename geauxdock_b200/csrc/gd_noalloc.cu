// gd_noalloc.cu -- pose energies without any memory allocation.
//
// Who needs this: callers that cannot call cudaMalloc/cudaFree around a
// docking call.  Examples: a host process whose device memory is owned by
// another allocator (a framework's caching allocator or a pool reserved at
// start-up), where a raw cudaMalloc would take memory that allocator has
// already accounted for; and latency-bound serving loops, where cudaFree
// synchronises the whole device and would stall every other stream's docking
// work.  gd_eval_poses() allocates device buffers for each call;
// gd_eval_poses_noalloc() does the same work with caller-provided device
// buffers for inputs and outputs, and keeps its own scratch (the packed
// device layout of the Complex, written by the device packer of
// gd_devpack.cu) in one fixed-size array declared below.
//
// The scratch array is a file-scope __device__ variable: every GPU that loads
// libgdock.so holds it (gd_noalloc_scratch_bytes(): 5.60 MiB) until the
// process exits.  Its size covers
// the reference Complex's own capacity (64 ligand atoms, 64 ligand
// conformations, 20 protein conformations of up to 2048 points, 10240 KDE
// points, 512 MCS rows); inputs beyond that are rejected with GD_E_CAPACITY.
// All calls on a device share the array and it keeps the last call's
// contents, so calls whose GPU work overlaps (different streams, or different
// host threads) race on it: issue them one after another.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "gd_device.cuh"
#include "gd_pack.h"

namespace gd {
namespace {

constexpr int kNaMaxDevices = 64;

// Layout of the scratch array: the packed job (gd_internal.h) at the largest
// size a reference Complex can describe.
struct NoAllocScratch {
  DevJob job;
  DevParams par;
  int err[4];     // flag, failure kind, field id, value (cleared at the start of every call)
  int2 lgrp[GD_MAXLIG];
  int ncdc[GD_MAX_CONF_PRT];
  float lcenter[GD_MAX_CONF_LIG * 3];
  float pcenter[GD_MAX_CONF_PRT * 3];
  float tcc[GD_MAX_MCS_ROW];
  float4 lig[GD_MAX_CONF_LIG * GD_MAXLIG];
  float4 kde[GD_MAXKDE];
  float4 mcs[GD_MAXLIG * GD_MAX_MCS_ROW];
  float4 pos[GD_MAX_CONF_PRT * GD_MAXPRO];
  float2 aux[GD_MAX_CONF_PRT * GD_MAXPRO];
  float psp[GD_MAX_CONF_PRT * kLigTypes * GD_MAXPRO];
  uint32_t pspmask[GD_MAX_CONF_PRT * GD_MAXPRO];
  float4 ref4[kLigTypes * kTabCols];
};

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {
std::mutex g_na_mu;
void *g_na_ptr[kNaMaxDevices] = {nullptr};

// The device packer's destination: the scratch array's members.
PackDst scratch_dst(NoAllocScratch *S)
{
  PackDst D{};
  D.job = &S->job;
  D.par = &S->par;
  D.ref4 = S->ref4;
  D.err = S->err;
  D.lgrp = S->lgrp;
  D.lcenter = S->lcenter;
  D.pcenter = S->pcenter;
  D.tcc = S->tcc;
  D.lig = S->lig;
  D.kde = S->kde;
  D.mcs = S->mcs;
  D.pos = S->pos;
  D.aux = S->aux;
  D.ncdc = S->ncdc;
  D.psp = S->psp;
  D.pspmask = S->pspmask;
  D.kde_cap = GD_MAXKDE;
  D.Ppad = 0;
  D.nkde_expect = -1;
  D.expect_L = D.expect_nlig = D.expect_nprt = D.expect_M = D.expect_ntmp = -1;
  D.rep = nullptr;
  return D;
}

}  // namespace
}  // namespace gd

using namespace gd;

// Set-up on the calling thread's current device: the device address of the
// scratch array, looked up once per device.  The first call on a device does
// this look-up; make that first call before any stream capture.
static int noalloc_scratch(NoAllocScratch **out)
{
  int dev = 0;
  GD_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) return fail(GD_E_INVALID, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(GD_E_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(e));
    g_na_ptr[dev] = p;
  }
  *out = (NoAllocScratch *)g_na_ptr[dev];
  return GD_OK;
}

extern "C" size_t gd_noalloc_scratch_bytes(void) { return sizeof(NoAllocScratch); }

extern "C" int gd_eval_poses_noalloc(const Complex *d_complex, int n, const int *d_conf, const float *d_mm,
                                     int precision, float *d_out, float *d_raw, void *stream)
{
  if (!d_complex || n < 0 || (n > 0 && (!d_conf || !d_mm || !d_out))) return fail(GD_E_INVALID, "null argument");
  if (precision < GD_PREC_FP32 || precision > GD_PREC_FP64) return fail(GD_E_INVALID, "precision = %d", precision);
  cudaStream_t st = (cudaStream_t)stream;
  int nsm = 0, dev = 0;
  GD_CUDA(cudaGetDevice(&dev));
  if (st != nullptr) {
    // the scratch address below is the current device's: the stream must belong to it
    int sdev = -1;
    GD_CUDA(cudaStreamGetDevice(st, &sdev));
    if (sdev != dev)
      return fail(GD_E_INVALID, "gd_eval_poses_noalloc: the stream belongs to device %d, the current device is %d",
                  sdev, dev);
  }
  NoAllocScratch *S = nullptr;
  GD_TRY(noalloc_scratch(&S));
  GD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  // the failure flag and its details must start at zero on every call
  GD_CUDA(cudaMemsetAsync(S->err, 0, sizeof(S->err), st));
  GD_CUDA(device_pack(d_complex, scratch_dst(S), st));
  const int grid = std::max(1, std::min((n + 7) / 8, nsm * 8));
  GD_CUDA(launch_eval_global(precision, &S->job, d_conf, d_mm, n, d_out, d_raw, &S->err[0], grid, st));
  int h[4] = {0, 0, 0, 0};
  GD_CUDA(cudaMemcpyAsync(h, S->err, sizeof(h), cudaMemcpyDeviceToHost, st));
  GD_CUDA(cudaStreamSynchronize(st));
  if (h[0] & kErrPack) {
    if (h[1] == kPackFailCapacity)
      return fail(GD_E_CAPACITY, "gd_eval_poses_noalloc: %s = %d exceeds the fixed scratch (%zu B, sized for the "
                                 "reference Complex caps)", pack_field_name(h[2]), h[3], sizeof(NoAllocScratch));
    return fail(GD_E_INVALID, "gd_eval_poses_noalloc: invalid %s: %d", pack_field_name(h[2]), h[3]);
  }
  if (h[0]) return fail(GD_E_INVALID, "gd_eval_poses_noalloc: a pose's conformation index is out of range");
  return GD_OK;
}
