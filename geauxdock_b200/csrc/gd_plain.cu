// gd_plain.cu -- the plain Monte Carlo kernel: the reference's own parallel
// structure, written for sm_100a.
//
// Structure of src/backend_gpu/kernel_cuda_l1_montecarlo.cu:29-536: one
// thread block per replica, a 2-D thread tile over (ligand atom, protein
// point) pairs with 8 ligand rows (bdy_prt = 8, :251), the pocket read from
// global memory through the read-only cache, the force-field tables copied to
// shared memory, block-wide reductions after every energy term, and the KDE
// term visiting every KDE point with a type test (energy_kde_v1.cu).  It uses
// the same packed data, Philox draws and FP64 Metropolis test as the batched
// kernel, so both produce the same trajectories up to FP32 rounding; it is
// the baseline the batched kernel is measured against.
#include "gd_device.cuh"
#include "gd_internal.h"

namespace gd {

namespace {

constexpr int kBD = 256;        // threads per block
constexpr int kBdy = 8;         // ligand rows of the PRT tile (kernel_cuda_l1_montecarlo.cu:251)
constexpr int kBdx = kBD / kBdy;  // 32 protein columns
constexpr int kWarps = kBD / 32;
constexpr float kLog2e = 1.4426950408889634f;
constexpr float kSqrt2PiInvNeg = -0.3989422804014327f;

__device__ __forceinline__ float block_sum(float v, float *red)
{
  v = warp_sum(v);
  const int w = threadIdx.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  if (threadIdx.x == 0)
    for (int i = 0; i < kWarps; ++i) s += red[i];
  return s;  // valid in thread 0
}

}  // namespace

__global__ void __launch_bounds__(kBD) plain_kernel(const DevJob *jobp, int s_begin, int nsteps, int flags,
                                                    const int *err)
{
  // a Complex the device packer refused (gd_devpack.cu) leaves its job unread
  if (err && (*(volatile const int *)err & kErrPack)) return;
  const DevJob &J = *jobp;
  __shared__ DevParams par;
  __shared__ float4 lig_s[kMaxAtoms];
  __shared__ int ltype_s[kMaxAtoms];
  __shared__ float red[kWarps];
  __shared__ float u_s[8];
  __shared__ float mmn_s[6];
  __shared__ float e_s[10];
  __shared__ ReplicaMC srep;
  __shared__ int acc_s;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int L = J.natom, P = J.npoint_pad, K = J.nkde, M = J.nmcs;
  {
    const float4 *src = reinterpret_cast<const float4 *>(J.par);
    float4 *dst = reinterpret_cast<float4 *>(&par);
    for (int i = tid; i < (int)(sizeof(DevParams) / 16); i += kBD) dst[i] = src[i];
    for (int a = tid; a < L; a += kBD) ltype_s[a] = J.lgrp[a].x;
  }
  __syncthreads();

  for (int r = blockIdx.x; r < J.nrep; r += gridDim.x) {
    const int gr = J.rid_base + r;
    if (tid < 32) reinterpret_cast<int *>(&srep)[tid] = reinterpret_cast<const int *>(J.rep + r)[tid];
    if (tid == 0) {
      acc_s = J.run_acc[r];
      if (J.rec && (flags & kMcResetRecord)) J.rec[r].next_entry = 0;
    }
    __syncthreads();
    const int ilig = srep.idx_lig, iprt = srep.idx_prt;
    const float *lc = J.lcenter + 3 * ilig;
    const float *pc = J.pcenter + 3 * iprt;
    const float4 *pos = J.pos + (size_t)iprt * P;
    const float2 *aux = J.aux + (size_t)iprt * P;
    const float *pspc = J.psp + (size_t)iprt * kLigTypes * P;
    const double mbeta = (double)J.minus_beta[srep.idx_tmp];
    const bool initial = (flags & kMcInitial) != 0;
    Record *rec = (J.rec && (flags & kMcRecord)) ? J.rec + r : nullptr;
    double st_sum = 0, st_sum2 = 0;
    long long st_acc = 0;

    for (int s = s_begin; s < s_begin + nsteps; ++s) {
      // record the old state, kernel_cuda_l1_montecarlo.cu:290-297
      if (acc_s) {
        if (tid == 0) srep.step = s;
        __syncthreads();
        if (rec && tid < 32) {
          const int ne = rec->next_entry;
          if (ne < GD_STEPS_PER_DUMP)
            reinterpret_cast<int *>(&rec->replica[ne])[tid] = reinterpret_cast<const int *>(&srep)[tid];
          __syncwarp();
          if (tid == 0) rec->next_entry = ne + 1;
        }
      }
      // move, kernel_cuda_l1_montecarlo.cu:307-328
      if (tid == 0) {
        float u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (!initial) {
          const Philox4 d0 = philox4x32_10((uint32_t)s, (uint32_t)gr, 0u, 0u, J.key0, J.key1);
          const Philox4 d1 = philox4x32_10((uint32_t)s, (uint32_t)gr, 0u, 1u, J.key0, J.key1);
          for (int i = 0; i < 4; ++i) {
            u[i] = u01(d0.v[i]);
            u[4 + i] = u01(d1.v[i]);
          }
        }
        for (int i = 0; i < 8; ++i) u_s[i] = u[i];
        for (int i = 0; i < 6; ++i) mmn_s[i] = __fmaf_rn(par.move_scale[i], u[i], srep.movematrix[i]);
      }
      __syncthreads();
      // rotation + translation (every thread builds the matrix; :336-380)
      {
        float s1, c1, s2, c2, s3, c3;
        sincosf(mmn_s[3], &s1, &c1);
        sincosf(mmn_s[4], &s2, &c2);
        sincosf(mmn_s[5], &s3, &c3);
        const float r00 = c1 * c2, r01 = c1 * s2 * s3 - c3 * s1, r02 = s1 * s3 + c1 * c3 * s2;
        const float r10 = c2 * s1, r11 = c1 * c3 + s1 * s2 * s3, r12 = c3 * s1 * s2 - c1 * s3;
        const float r20 = -s2, r21 = c2 * s3, r22 = c2 * c3;
        const float tx = mmn_s[0] + lc[0], ty = mmn_s[1] + lc[1], tz = mmn_s[2] + lc[2];
        const float4 *lsrc = J.lig + (size_t)ilig * J.lstride;
        for (int a = tid; a < L; a += kBD) {
          const float4 v = lsrc[a];
          lig_s[a] = make_float4(r00 * v.x + r01 * v.y + r02 * v.z + tx, r10 * v.x + r11 * v.y + r12 * v.z + ty,
                                 r20 * v.x + r21 * v.y + r22 * v.z + tz, v.w);
        }
      }
      __syncthreads();

      // PRT, energy_prt_v1.cu: 2-D tile, ty = ligand row, tx = protein column
      const int ty = tid / kBdx, tx = tid % kBdx;
      float evdw = 0, eele = 0, epmf = 0, epsp = 0, ehdb = 0, ehpc = 0;
      for (int j = 0; j < L; j += kBdy) {
        const int l = j + ty;
        float ehpc1 = 0.f;
        if (l < L) {
          const float4 la = lig_s[l];
          const int lt = ltype_s[l];
          for (int p = tx; p < P; p += kBdx) {
            const float4 q = __ldg(pos + p);
            const float2 w = __ldg(aux + p);
            const int pt = __float_as_int(w.y);
            const float dx = la.x - q.x, dy = la.y - q.y, dz = la.z - q.z;
            const float d2 = dx * dx + dy * dy + dz * dz;
            const float d4 = d2 * d2;
            const float d = sqrtf(d2);
            const float hp = 1.0f - (3.5f / 81.0f * d2 - 4.5f / 81.0f / 81.0f * d4 +
                                     2.5f / 81.0f / 81.0f / 81.0f * d4 * d2 -
                                     0.5f / 81.0f / 81.0f / 81.0f / 81.0f * d4 * d4);
            ehpc1 += (d2 <= 81.0f) ? w.x * hp : 0.0f;
            const float4 t4 = par.tab4[lt][pt];                       // pmf0, pmf1 in .z, .w
            const float4 rf = __ldg(J.ref4 + lt * kTabCols + pt);   // p1a, p2a, hdb0, hdb1
            const float2 t2 = make_float2(rf.z, rf.w);
            const float p1 = __fdividef(rf.x, d4 * d4 * d);
            const float p2 = __fdividef(rf.y, d4 * d2);
            const float p4 = p1 * par.lj0 * (1.0f + par.lj1 * d2) + 1.0f;
            evdw += __fdividef(p1 - p2, p4);
            const float s1 = par.el1 * d;
            const float g1 = (s1 < 1.0f) ? (par.el0 + par.a1 * s1 * s1 + par.b1 * s1 * s1 * s1) : __fdividef(1.0f, s1);
            eele += la.w * q.w * g1;
            const float dmp = d + t4.z;                               // t4.z = -pmf0
            epmf += __fdividef(t4.w, 1.0f + __expf((-0.5f * d + 6.0f) * dmp));
            if (dmp <= 0.0f) epsp += __ldg(pspc + (size_t)lt * P + p);
            if (t2.x > 0.1f) {
              const float h3 = (d - t2.x) * t2.y;
              ehdb += t2.y * __expf(-0.5f * h3 * h3);
            }
          }
        }
        // hydrophobic restraint per ligand row (one warp per row)
        ehpc1 = warp_sum(ehpc1);
        if (lane == 0 && l < L) {
          const int lt = ltype_s[l];
          const float h2 = (ehpc1 - par.hpl0[lt]) / par.hpl1[lt];
          ehpc += 0.5f * h2 * h2 - par.hpl2[lt];
        }
      }
      const float bvdw = block_sum(evdw, red);
      const float bele = block_sum(eele, red);
      const float bpmf = block_sum(epmf, red);
      const float bpsp = block_sum(epsp, red);
      const float bhdb = block_sum(ehdb, red);
      const float bhpc = block_sum(ehpc, red);

      // KDE v1: every KDE point visited, same-type test (energy_kde_v1.cu:189-270)
      float ekde = 0.f;
      for (int j = 0; j < L; j += kBdy) {
        const int l = j + ty;
        float k1 = 0.f;
        int k2 = 0;
        if (l < L) {
          const float4 la = lig_s[l];
          const int lt = ltype_s[l];
          for (int k = tx; k < K; k += kBdx) {
            const float4 q = __ldg(J.kde + k);
            if (__float_as_int(q.w) == lt) {
              const float dx = la.x - q.x, dy = la.y - q.y, dz = la.z - q.z;
              k1 += ex2_approx(par.kde2 * kLog2e * (dx * dx + dy * dy + dz * dz));
              ++k2;
            }
          }
        }
        k1 = warp_sum(k1);
        k2 = warp_sum(k2);
        if (lane == 0 && l < L && k2 != 0) ekde += k1 / (float)k2;
      }
      const float bkde = block_sum(ekde, red);

      // MCS, energy_mcs_v1.cu: rows over ty, atoms over tx
      float elhm = 0.f;
      for (int j = 0; j < M; j += kBdy) {
        const int m = j + ty;
        float s = 0.f;
        int n = 0;
        if (m < M) {
          for (int l = tx; l < L; l += kBdx) {
            const float4 q = __ldg(J.mcs + (size_t)l * M + m);
            if (q.w != 0.0f) {
              const float4 la = lig_s[l];
              const float dx = la.x - q.x, dy = la.y - q.y, dz = la.z - q.z;
              s += dx * dx + dy * dy + dz * dz;
              ++n;
            }
          }
        }
        s = warp_sum(s);
        n = warp_sum(n);
        if (lane == 0 && m < M) elhm += __ldg(J.tcc + m) * sqrtf(s / (float)n);
      }
      const float blhm = block_sum(elhm, red);

      if (tid == 0) {
        float r9[9];
        r9[0] = bvdw;
        r9[1] = bele;
        r9[2] = bpmf;
        r9[3] = bpsp;
        r9[4] = bhdb * kSqrt2PiInvNeg;
        r9[5] = bhpc;
        r9[6] = bkde * par.kde3_inv;
        r9[7] = logf(blhm / (float)M);
        float dst = 0.f;
        for (int i = 0; i < 3; ++i) {
          const float t = (lc[i] + mmn_s[i]) - pc[i];
          dst += t * t;
        }
        r9[8] = sqrtf(dst);
        float tot = 0.f;
        for (int i = 0; i < 9; ++i) {
          float v = r9[i];
          if (i < 7) v = v / (float)L;
          v = par.a_para[i] * v + par.b_para[i];
          e_s[i] = v;
          tot += par.w[i] * v;
        }
        e_s[9] = tot;
        int accept = 1;
        if (!initial) {
          const double lr = ((double)tot - (double)srep.energy[9]) * mbeta;
          accept = log((double)u_s[6]) < lr;
        }
        if (accept) {
          for (int i = 0; i < 10; ++i) srep.energy[i] = e_s[i];
          for (int i = 0; i < 6; ++i) srep.movematrix[i] = mmn_s[i];
        }
        st_acc += accept;
        st_sum += (double)srep.energy[9];
        st_sum2 += (double)srep.energy[9] * (double)srep.energy[9];
        acc_s = accept;
      }
      __syncthreads();
    }
    if (tid == 0) {
      J.run_acc[r] = acc_s;
      if (flags & kMcStoreAccept) srep.is_accept = acc_s;
      RepStats &S = J.stats[r];
      S.e_sum += st_sum;
      S.e_sum2 += st_sum2;
      S.n_steps += nsteps;
      S.n_accept += st_acc;
    }
    __syncthreads();
    if (tid < 32) reinterpret_cast<int *>(J.rep + r)[tid] = reinterpret_cast<const int *>(&srep)[tid];
    __syncthreads();
  }
}

cudaError_t launch_plain(const DevJob *d_job, int nrep, int s_begin, int nsteps, int flags, int *d_err,
                         cudaStream_t st)
{
  if (nrep <= 0) return cudaSuccess;
  plain_kernel<<<nrep, kBD, 0, st>>>(d_job, s_begin, nsteps, flags, d_err);
  return cudaGetLastError();
}

}  // namespace gd
