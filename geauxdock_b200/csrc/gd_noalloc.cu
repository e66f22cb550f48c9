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
// device layout of the Complex) in one fixed-size array declared below.
//
// The scratch array is a file-scope __device__ variable: every GPU that loads
// libgdock.so holds it (gd_noalloc_scratch_bytes(): 5.60 MiB) until the process exits.  Its size covers
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
constexpr int kNaFailCapacity = 1;   // a size beyond the scratch
constexpr int kNaFailInput = 2;      // a malformed value (type, index, empty MCS row)

// Layout of the scratch array: the packed job (gd_internal.h) at the largest
// size a reference Complex can describe.
struct NoAllocScratch {
  DevJob job;
  DevParams par;
  int err;        // nonzero: the call failed (cleared at the start of every call)
  int info[3];    // first failure: kind, field id, value
  int ltype[GD_MAXLIG];
  int2 lgrp[GD_MAXLIG];
  int perm[GD_MAXLIG];
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

// field ids reported in info[1]
enum { kFieldNLig = 1, kFieldNPrt, kFieldNatom, kFieldNatomConf, kFieldNpoint, kFieldKde, kFieldMcs, kFieldLigType,
       kFieldPrtType, kFieldSeq3r, kFieldMcsRow, kFieldP1a };

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

__device__ void na_fail(NoAllocScratch *S, int kind, int field, int value)
{
  if (atomicCAS(&S->info[0], 0, kind) == 0) {
    S->info[1] = field;
    S->info[2] = value;
  }
  atomicOr(&S->err, 1);
}

__device__ __forceinline__ float na_as_float(int i) { return __int_as_float(i); }

// Sizes, validation, force-field tables, ligand atom order, KDE points sorted
// by type with per-type ranges, and the DevJob header.  One CTA of 256 threads.
__global__ void na_setup_kernel(const Complex *__restrict__ cx, NoAllocScratch *S)
{
  __shared__ int s_ok, s_L, s_P, s_K, s_M, s_nlig, s_nprt;
  __shared__ int s_kcnt[kLigTypes], s_kbeg[kLigTypes];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    const int nlig = cx->size.n_lig, nprt = cx->size.n_prt, K = cx->size.kde_npoint, M = cx->size.mcs_nrow;
    const int L = cx->lig[0].lig_natom;
    int ok = 1, P = 0;
    if (nlig < 1 || nlig > GD_MAX_CONF_LIG) na_fail(S, nlig < 1 ? kNaFailInput : kNaFailCapacity, kFieldNLig, nlig), ok = 0;
    else if (nprt < 1 || nprt > GD_MAX_CONF_PRT) na_fail(S, nprt < 1 ? kNaFailInput : kNaFailCapacity, kFieldNPrt, nprt), ok = 0;
    else if (L < 1 || L > GD_MAXLIG) na_fail(S, L < 1 ? kNaFailInput : kNaFailCapacity, kFieldNatom, L), ok = 0;
    else if (K < 0 || K > GD_MAXKDE) na_fail(S, K < 0 ? kNaFailInput : kNaFailCapacity, kFieldKde, K), ok = 0;
    else if (M < 1 || M > GD_MAX_MCS_ROW) na_fail(S, M < 1 ? kNaFailInput : kNaFailCapacity, kFieldMcs, M), ok = 0;
    if (ok)
      for (int i = 0; i < nlig; ++i)
        if (cx->lig[i].lig_natom != L) {
          na_fail(S, kNaFailInput, kFieldNatomConf, i);
          ok = 0;
          break;
        }
    if (ok)
      for (int i = 0; i < nprt; ++i) {
        const int n = cx->prt[i].prt_npoint;
        if (n < 1 || n > GD_MAXPRO) {
          na_fail(S, n < 1 ? kNaFailInput : kNaFailCapacity, kFieldNpoint, n);
          ok = 0;
          break;
        }
        P = max(P, n);
      }
    s_ok = ok;
    s_L = L;
    s_P = P;
    s_K = K;
    s_M = M;
    s_nlig = nlig;
    s_nprt = nprt;
  }
  __syncthreads();
  if (!s_ok) return;
  const int L = s_L, K = s_K, M = s_M, nlig = s_nlig, nprt = s_nprt;

  // type and index validation
  for (int a = tid; a < L; a += blockDim.x) {
    const int t = cx->lig[0].t2[a];
    if (t < 0 || t >= kLigTypes) na_fail(S, kNaFailInput, kFieldLigType, a);
  }
  for (int q = tid; q < nprt * GD_MAXPRO; q += blockDim.x) {
    const int i = q / GD_MAXPRO, k = q % GD_MAXPRO;
    const Protein &pr = cx->prt[i];
    if (k >= pr.prt_npoint) continue;
    if (pr.t[k] < 0 || pr.t[k] >= kPadType) na_fail(S, kNaFailInput, kFieldPrtType, k);
    if (pr.c[k] == 2 && (pr.seq3r[k] < 0 || pr.seq3r[k] >= GD_MAXPRO)) na_fail(S, kNaFailInput, kFieldSeq3r, k);
  }

  // force-field tables, as the host packer's build_params
  const EnePara &ep = cx->enepara;
  DevParams &par = S->par;
  for (int q = tid; q < kLigTypes * kTabCols; q += blockDim.x) {
    const int lt = q / kTabCols, pt = q % kTabCols;
    if (pt < kPadType) {
      if (!(ep.p1a[lt][pt] > 0.f)) na_fail(S, kNaFailInput, kFieldP1a, q);
      par.tab4[lt][pt] = tab4_entry(ep.p1a[lt][pt], ep.p2a[lt][pt], ep.pmf0[lt][pt], ep.pmf1[lt][pt]);
      const float h0 = ep.hdb0[lt][pt], h1 = ep.hdb1[lt][pt];
      const bool on = h0 > 0.1f;
      par.tab2[lt][pt] = on ? make_float2((float)((double)h1 * kHdbC), (float)(-(double)h0 * (double)h1 * kHdbC))
                            : make_float2(0.f, 0.f);
      S->ref4[q] = make_float4(ep.p1a[lt][pt], ep.p2a[lt][pt], on ? h0 : 0.f, on ? h1 : 0.f);
    } else {
      par.tab4[lt][pt] = tab4_padding();
      par.tab2[lt][pt] = make_float2(0.f, 0.f);
      S->ref4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  for (int q = tid; q < kLigTypes; q += blockDim.x) {
    par.hpl0[q] = ep.hpl0[q];
    par.hpl1[q] = ep.hpl1[q];
    par.hpl2[q] = ep.hpl2[q];
    uint32_t m = 0;
    for (int pt = 0; pt < kPadType; ++pt) m |= (ep.hdb0[q][pt] > 0.1f ? 1u : 0u) << pt;
    par.hdbmask[q] = m;
  }
  for (int q = tid; q < 12; q += blockDim.x) {
    par.a_para[q] = q < GD_MAXWEI ? ep.a_para[q] : 0.f;
    par.b_para[q] = q < GD_MAXWEI ? ep.b_para[q] : 0.f;
    par.w[q] = q < GD_MAXWEI ? ep.w[q] : 0.f;
  }
  if (tid == 0) {
    par.lj0 = ep.lj0;
    par.lj1 = ep.lj1;
    par.el0 = ep.el0;
    par.el1 = ep.el1;
    par.inv_el1 = 1.0f / ep.el1;
    par.a1 = ep.a1;
    par.b1 = ep.b1;
    par.kde2 = ep.kde2;
    par.kde3_inv = 1.0f / ep.kde3;
    par.lj01 = (float)((double)ep.lj0 * ep.lj1);
    par.ele_a = (float)((double)ep.a1 * ep.el1 * ep.el1);
    par.ele_b = (float)((double)ep.b1 * ep.el1 * ep.el1 * ep.el1);
    par.ele_d2max = (float)(1.0 / ((double)ep.el1 * ep.el1));
    par.hdb_cinv = (float)(1.0 / kHdbC);
    for (int i = 0; i < 6; ++i) par.move_scale[i] = cx->mcpara.move_scale[i];
    par.kde3 = ep.kde3;
    par.pad_ = 0.f;
    // ligand atoms grouped by type, stable (the host packer's order)
    int k = 0;
    for (int t = 0; t < kLigTypes; ++t)
      for (int a = 0; a < L; ++a)
        if (cx->lig[0].t2[a] == t) {
          S->perm[k] = a;
          S->ltype[k] = t;
          ++k;
        }
    int end = L;
    for (int a = L - 1; a >= 0; --a) {
      if (a + 1 < L && S->ltype[a + 1] != S->ltype[a]) end = a + 1;
      S->lgrp[a] = make_int2(S->ltype[a], end);
    }
  }
  for (int q = tid; q < nlig * 3; q += blockDim.x) S->lcenter[q] = cx->lig[q / 3].center[q % 3];
  for (int q = tid; q < nprt * 3; q += blockDim.x) S->pcenter[q] = cx->prt[q / 3].pocket_center[q % 3];
  for (int q = tid; q < M; q += blockDim.x) S->tcc[q] = cx->mcs[q].tcc;

  // KDE points of ligand types, sorted by type (stable): count, prefix, scatter
  const int nwarps = blockDim.x >> 5;
  for (int t = warp; t < kLigTypes; t += nwarps) {
    int cnt = 0;
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      cnt += __popc(__ballot_sync(0xffffffffu, k < K && cx->kde.t[k] == t));
    }
    if (lane == 0) s_kcnt[t] = cnt;
  }
  __syncthreads();
  if (tid == 0) {
    int b = 0;
    for (int t = 0; t < kLigTypes; ++t) {
      s_kbeg[t] = s_kcnt[t] ? b : 0;
      b += s_kcnt[t];
    }
  }
  __syncthreads();
  for (int t = warp; t < kLigTypes; t += nwarps) {
    int at = s_kbeg[t];
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      const bool m = k < K && cx->kde.t[k] == t;
      const unsigned b = __ballot_sync(0xffffffffu, m);
      if (m) {
        const int o = at + __popc(b & ((1u << lane) - 1u));
        S->kde[o] = make_float4(cx->kde.x[k], cx->kde.y[k], cx->kde.z[k], na_as_float(t));
      }
      at += __popc(b);
    }
  }
  __syncthreads();
  if (tid == 0) {
    DevJob &J = S->job;
    J.natom = L;
    J.nlig = nlig;
    J.lstride = (L + 3) & ~3;
    J.lig = S->lig;
    J.lgrp = S->lgrp;
    J.lcenter = S->lcenter;
    J.npoint_pad = ((s_P + kPointAlign - 1) / kPointAlign) * kPointAlign;
    J.nprt = nprt;
    J.pos = S->pos;
    J.aux = S->aux;
    J.ncdc = S->ncdc;
    J.pcenter = S->pcenter;
    J.psp = S->psp;
    J.pspmask = S->pspmask;
    int nk = 0;
    for (int t = 0; t < kLigTypes; ++t) {
      J.kbeg[t] = s_kbeg[t];
      J.kcnt[t] = s_kcnt[t];
      nk += s_kcnt[t];
    }
    J.nkde = nk;
    J.kde = S->kde;
    J.nmcs = M;
    J.mcs = S->mcs;
    J.tcc = S->tcc;
    J.ntmp = 0;
    J.minus_beta = nullptr;
    J.par = &S->par;
    J.ref4 = S->ref4;
    J.nrep = 0;
    J.rep = nullptr;
    J.run_acc = nullptr;
    J.stats = nullptr;
    J.rec = nullptr;
    J.key0 = J.key1 = 0;
    J.rid_base = 0;
    J.nrep_total = 0;
  }
}

// One CTA per protein conformation.  Points are ordered as the host packer
// orders them: hydrophobic-contact (cdc == 1) points first, each part sorted
// by point type (stable); 60 buckets (cdc, type), two per warp, counted and
// scattered with warp ballots.  Padding with inert points; pocket-specific
// potential gathered with its non-zero type mask.
__global__ void __launch_bounds__(1024) na_pocket_kernel(const Complex *__restrict__ cx, NoAllocScratch *S)
{
  constexpr int kBuckets = 2 * kPadType;
  __shared__ int s_cnt[kBuckets], s_beg[kBuckets];
  if (S->err) return;
  const int i = blockIdx.x;
  const DevJob &J = S->job;
  if (i >= J.nprt) return;
  const Protein &pr = cx->prt[i];
  const int np = pr.prt_npoint, Pp = J.npoint_pad;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  auto bucket = [&](int k) { return (pr.cdc[k] == 1 ? 0 : kPadType) + pr.t[k]; };
  for (int bk = warp; bk < kBuckets; bk += nwarps) {
    int cnt = 0;
    for (int k0 = 0; k0 < np; k0 += 32) {
      const int k = k0 + lane;
      cnt += __popc(__ballot_sync(0xffffffffu, k < np && bucket(k) == bk));
    }
    if (lane == 0) s_cnt[bk] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int b = 0;
    for (int q = 0; q < kBuckets; ++q) {
      s_beg[q] = b;
      b += s_cnt[q];
    }
    int nc = 0;
    for (int q = 0; q < kPadType; ++q) nc += s_cnt[q];
    S->ncdc[i] = nc;
  }
  __syncthreads();
  float4 *pos = S->pos + (size_t)i * Pp;
  float2 *aux = S->aux + (size_t)i * Pp;
  float *psp = S->psp + (size_t)i * kLigTypes * Pp;
  uint32_t *pm = S->pspmask + (size_t)i * Pp;
  for (int bk = warp; bk < kBuckets; bk += nwarps) {
    int at = s_beg[bk];
    for (int k0 = 0; k0 < np; k0 += 32) {
      const int k = k0 + lane;
      const bool m = k < np && bucket(k) == bk;
      const unsigned b = __ballot_sync(0xffffffffu, m);
      if (m) {
        const int j = at + __popc(b & ((1u << lane) - 1u));
        pos[j] = make_float4(pr.x[k], pr.y[k], pr.z[k], pr.ele[k]);
        aux[j] = make_float2(pr.cdc[k] == 1 ? pr.hpp[k] : 0.f, na_as_float(pr.t[k]));
        const bool c2 = pr.c[k] == 2;
        const int col = pr.seq3r[k];
        uint32_t mask = 0;
        for (int lt = 0; lt < kLigTypes; ++lt) {
          const float v = c2 ? cx->psp.psp[lt][col] : 0.f;
          psp[(size_t)lt * Pp + j] = v;
          mask |= (v != 0.f ? 1u : 0u) << lt;
        }
        pm[j] = mask;
      }
      at += __popc(b);
    }
  }
  for (int j = np + threadIdx.x; j < Pp; j += blockDim.x) {
    pos[j] = make_float4(1.0e4f + (float)j, 1.0e4f, 1.0e4f, 0.f);
    aux[j] = make_float2(0.f, na_as_float(kPadType));
    pm[j] = 0u;
    for (int lt = 0; lt < kLigTypes; ++lt) psp[(size_t)lt * Pp + j] = 0.f;
  }
}

// Ligand conformations in grouped atom order, MCS templates atom-major.
__global__ void na_ligand_kernel(const Complex *__restrict__ cx, NoAllocScratch *S)
{
  if (S->err) return;
  const DevJob &J = S->job;
  const int L = J.natom, M = J.nmcs, ls = J.lstride;
  const int stride = gridDim.x * blockDim.x;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  for (int q = g; q < J.nlig * ls; q += stride) {
    const int i = q / ls, a = q % ls;
    if (a < L) {
      const int s = S->perm[a];
      const Ligand &lg = cx->lig[i];
      S->lig[q] = make_float4(lg.x2[s], lg.y2[s], lg.z2[s], cx->lig[0].c2[s]);
    } else {
      S->lig[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  for (int q = g; q < L * M; q += stride) {
    const int a = q / M, m = q % M;
    const int s = S->perm[a];
    const float x = cx->mcs[m].x[s];
    S->mcs[q] = make_float4(x, cx->mcs[m].y[s], cx->mcs[m].z[s], x != GD_MCS_INVALID_COORD ? 1.f : 0.f);
  }
  for (int m = g; m < M; m += stride) {
    int n = 0;
    for (int a = 0; a < L; ++a) n += cx->mcs[m].x[a] != GD_MCS_INVALID_COORD;
    if (n == 0) na_fail(S, kNaFailInput, kFieldMcsRow, m);
  }
}

std::mutex g_na_mu;
void *g_na_ptr[kNaMaxDevices] = {nullptr};

const char *field_name(int f)
{
  switch (f) {
    case kFieldNLig: return "size.n_lig (ligand conformations)";
    case kFieldNPrt: return "size.n_prt (protein conformations)";
    case kFieldNatom: return "lig[0].lig_natom (ligand atoms)";
    case kFieldNatomConf: return "a ligand conformation's lig_natom (differs from conformation 0)";
    case kFieldNpoint: return "prt[i].prt_npoint (protein points)";
    case kFieldKde: return "size.kde_npoint (KDE points)";
    case kFieldMcs: return "size.mcs_nrow (MCS rows)";
    case kFieldLigType: return "a ligand atom type (index given)";
    case kFieldPrtType: return "a protein point type (index given)";
    case kFieldSeq3r: return "a class-2 point's seq3r (index given)";
    case kFieldMcsRow: return "an MCS row without any coordinate (row given)";
    case kFieldP1a: return "enepara.p1a <= 0 (index lt * 32 + pt given; the pair kernel needs p1a > 0)";
    default: return "unknown field";
  }
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
  GD_CUDA(cudaMemsetAsync(&S->err, 0, sizeof(int) * 4, st));
  na_setup_kernel<<<1, 256, 0, st>>>(d_complex, S);
  GD_CUDA(cudaGetLastError());
  na_pocket_kernel<<<GD_MAX_CONF_PRT, 1024, 0, st>>>(d_complex, S);
  GD_CUDA(cudaGetLastError());
  na_ligand_kernel<<<64, 256, 0, st>>>(d_complex, S);
  GD_CUDA(cudaGetLastError());
  const int grid = std::max(1, std::min((n + 7) / 8, nsm * 8));
  GD_CUDA(launch_eval_global(precision, &S->job, d_conf, d_mm, n, d_out, d_raw, &S->err, grid, st));
  int h[4] = {0, 0, 0, 0};
  GD_CUDA(cudaMemcpyAsync(h, &S->err, sizeof(h), cudaMemcpyDeviceToHost, st));
  GD_CUDA(cudaStreamSynchronize(st));
  if (h[0]) {
    if (h[1] == kNaFailCapacity)
      return fail(GD_E_CAPACITY, "gd_eval_poses_noalloc: %s = %d exceeds the fixed scratch (%zu B, sized for the "
                                 "reference Complex caps)", field_name(h[2]), h[3], sizeof(NoAllocScratch));
    if (h[1] == kNaFailInput) return fail(GD_E_INVALID, "gd_eval_poses_noalloc: invalid %s: %d", field_name(h[2]), h[3]);
    return fail(GD_E_INVALID, "gd_eval_poses_noalloc: a pose's conformation index is out of range");
  }
  return GD_OK;
}
