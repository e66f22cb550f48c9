// gd_devpack.cu -- packing a reference-layout Complex that is already in
// device memory into the kernels' structure-of-arrays layout, on the GPU.
//
// The same work as the host packer (gd_pack.cu: the semantics of the
// reference's OptimizeLigand / OptimizeProtein / OptimizePsp / OptimizeKde /
// OptimizeMcs / OptimizeEnepara, src/frontend/util_optimize_soa.C:37-540),
// with the same orders, so that both packings of one Complex are identical
// byte for byte:
//   - ligand atoms grouped by type, stable (util_optimize_soa.C:112-126), the
//     types with a hydrogen-bond parameter first;
//   - pocket points with the hydrophobic-contact flag first; in each part the
//     point types with a hydrogen-bond parameter first, each group sorted by
//     point type, stable; padded with inert points (type 30, far away);
//   - KDE points of ligand types sorted by type, stable, with per-type ranges
//     (util_optimize_soa.C:336-372; points of other types cannot match);
//   - MCS templates atom-major in grouped order, validity as energy_mcs_v1.cu;
//   - pocket-specific potential gathered per sorted class-2 point.
// Two callers: the allocation-free pose evaluation (destination: one static
// scratch array, gd_noalloc.cu) and Dock's refill of its resident state after
// CopyH2D put the next Complex on the GPU (destination: the arenas of the
// cached ensemble, gd_api.cu).  Invalid input sets the destination's error
// words and no header is written; the kernels downstream check the flag.
#include "gd_pack.h"

namespace gd {
namespace {

__device__ void dp_fail(const PackDst &D, int kind, int field, int value)
{
  if (atomicCAS(&D.err[1], 0, kind) == 0) {
    D.err[2] = field;
    D.err[3] = value;
  }
  atomicOr(&D.err[0], kErrPack);
}

__device__ __forceinline__ float dp_as_float(int i) { return __int_as_float(i); }

// The host packer's order of the ligand type groups: the types with a
// hydrogen-bond parameter for some point type first, each part by type.
__device__ void dp_ligand_type_order(const Complex *cx, int *order)
{
  uint32_t m = 0;
  for (int lt = 0; lt < kLigTypes; ++lt)
    for (int pt = 0; pt < kPadType; ++pt)
      if (cx->enepara.hdb0[lt][pt] > 0.1f) m |= 1u << lt;
  int q = 0;
  for (int t = 0; t < kLigTypes; ++t)
    if ((m >> t) & 1u) order[q++] = t;
  for (int t = 0; t < kLigTypes; ++t)
    if (!((m >> t) & 1u)) order[q++] = t;
}

// Ligand atoms grouped by type in that order (stable): perm[k] = input index
// of grouped atom k.
__device__ void dp_ligand_order(const Complex *cx, int L, int *perm, int *ltype)
{
  int order[kLigTypes];
  dp_ligand_type_order(cx, order);
  int k = 0;
  for (int q = 0; q < kLigTypes; ++q) {
    const int t = order[q];
    for (int a = 0; a < L; ++a)
      if (cx->lig[0].t2[a] == t) {
        perm[k] = a;
        ltype[k] = t;
        ++k;
      }
  }
}

// Sizes, validation, force-field tables, ligand atom order, KDE points sorted
// by type with per-type ranges, and (when everything is valid) the DevJob
// header.  One CTA of 256 threads.
__global__ void dp_setup_kernel(const Complex *__restrict__ cx, PackDst D)
{
  __shared__ int s_ok, s_L, s_P, s_K, s_M, s_nlig, s_nprt, s_ntmp, s_nk;
  __shared__ int s_kcnt[kLigTypes], s_kbeg[kLigTypes];
  __shared__ int s_perm[GD_MAXLIG], s_ltype[GD_MAXLIG];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    const int nlig = cx->size.n_lig, nprt = cx->size.n_prt, K = cx->size.kde_npoint, M = cx->size.mcs_nrow;
    const int ntmp = cx->size.n_tmp;
    const int L = cx->lig[0].lig_natom;
    int ok = 1, P = 0;
    if (nlig < 1 || nlig > GD_MAX_CONF_LIG) dp_fail(D, nlig < 1 ? kPackFailInput : kPackFailCapacity, kFieldNLig, nlig), ok = 0;
    else if (nprt < 1 || nprt > GD_MAX_CONF_PRT) dp_fail(D, nprt < 1 ? kPackFailInput : kPackFailCapacity, kFieldNPrt, nprt), ok = 0;
    else if (L < 1 || L > GD_MAXLIG) dp_fail(D, L < 1 ? kPackFailInput : kPackFailCapacity, kFieldNatom, L), ok = 0;
    else if (K < 0 || K > GD_MAXKDE) dp_fail(D, K < 0 ? kPackFailInput : kPackFailCapacity, kFieldKde, K), ok = 0;
    else if (M < 1 || M > GD_MAX_MCS_ROW) dp_fail(D, M < 1 ? kPackFailInput : kPackFailCapacity, kFieldMcs, M), ok = 0;
    else if (D.rep && (ntmp < 1 || ntmp > GD_MAX_TMP)) dp_fail(D, kPackFailInput, kFieldNTmp, ntmp), ok = 0;
    if (ok)
      for (int i = 0; i < nlig; ++i)
        if (cx->lig[i].lig_natom != L) {
          dp_fail(D, kPackFailInput, kFieldNatomConf, i);
          ok = 0;
          break;
        }
    if (ok)
      for (int i = 0; i < nprt; ++i) {
        const int n = cx->prt[i].prt_npoint;
        if (n < 1 || n > GD_MAXPRO) {
          dp_fail(D, n < 1 ? kPackFailInput : kPackFailCapacity, kFieldNpoint, n);
          ok = 0;
          break;
        }
        P = max(P, n);
      }
    const int Ppad = ((P + kPointAlign - 1) / kPointAlign) * kPointAlign;
    if (ok && D.Ppad > 0 && Ppad != D.Ppad) dp_fail(D, kPackFailShape, kFieldNpoint, P), ok = 0;
    if (ok && D.expect_L >= 0 && L != D.expect_L) dp_fail(D, kPackFailShape, kFieldNatom, L), ok = 0;
    if (ok && D.expect_nlig >= 0 && nlig != D.expect_nlig) dp_fail(D, kPackFailShape, kFieldNLig, nlig), ok = 0;
    if (ok && D.expect_nprt >= 0 && nprt != D.expect_nprt) dp_fail(D, kPackFailShape, kFieldNPrt, nprt), ok = 0;
    if (ok && D.expect_M >= 0 && M != D.expect_M) dp_fail(D, kPackFailShape, kFieldMcs, M), ok = 0;
    if (ok && D.rep && D.expect_ntmp >= 0 && ntmp != D.expect_ntmp) dp_fail(D, kPackFailShape, kFieldNTmp, ntmp), ok = 0;
    if (ok && D.rep && (D.rep_begin < 0 || D.rep_begin + D.nrep > cx->size.n_rep))
      dp_fail(D, kPackFailShape, kFieldReplica, D.rep_begin + D.nrep), ok = 0;
    s_ok = ok;
    s_L = L;
    s_P = D.Ppad > 0 ? D.Ppad : Ppad;
    s_K = K;
    s_M = M;
    s_nlig = nlig;
    s_nprt = nprt;
    s_ntmp = ntmp;
  }
  __syncthreads();
  if (!s_ok) return;
  const int L = s_L, K = s_K, M = s_M, nlig = s_nlig, nprt = s_nprt;

  // type and index validation
  for (int a = tid; a < L; a += blockDim.x) {
    const int t = cx->lig[0].t2[a];
    if (t < 0 || t >= kLigTypes) dp_fail(D, kPackFailInput, kFieldLigType, a);
  }
  for (int q = tid; q < nprt * GD_MAXPRO; q += blockDim.x) {
    const int i = q / GD_MAXPRO, k = q % GD_MAXPRO;
    const Protein &pr = cx->prt[i];
    if (k >= pr.prt_npoint) continue;
    if (pr.t[k] < 0 || pr.t[k] >= kPadType) dp_fail(D, kPackFailInput, kFieldPrtType, k);
    if (pr.c[k] == 2 && (pr.seq3r[k] < 0 || pr.seq3r[k] >= GD_MAXPRO)) dp_fail(D, kPackFailInput, kFieldSeq3r, k);
  }
  for (int m = tid; m < M; m += blockDim.x) {
    int n = 0;
    for (int a = 0; a < L; ++a) n += cx->mcs[m].x[a] != GD_MCS_INVALID_COORD;
    if (n == 0) dp_fail(D, kPackFailInput, kFieldMcsRow, m);
  }

  // force-field tables, as the host packer's build_params
  const EnePara &ep = cx->enepara;
  DevParams &par = *D.par;
  for (int q = tid; q < kLigTypes * kTabCols; q += blockDim.x) {
    const int lt = q / kTabCols, pt = q % kTabCols;
    if (pt < kPadType) {
      if (!(ep.p1a[lt][pt] > 0.f)) dp_fail(D, kPackFailInput, kFieldP1a, q);
      par.tab4[lt][pt] = tab4_entry(ep.p1a[lt][pt], ep.p2a[lt][pt], ep.pmf0[lt][pt], ep.pmf1[lt][pt]);
      const float h0 = ep.hdb0[lt][pt], h1 = ep.hdb1[lt][pt];
      const bool on = h0 > 0.1f;
      par.tab2[lt][pt] = on ? make_float2((float)((double)h1 * kHdbC), (float)(-(double)h0 * (double)h1 * kHdbC))
                            : make_float2(0.f, 0.f);
      D.ref4[q] = make_float4(ep.p1a[lt][pt], ep.p2a[lt][pt], on ? h0 : 0.f, on ? h1 : 0.f);
    } else {
      par.tab4[lt][pt] = tab4_padding();
      par.tab2[lt][pt] = make_float2(0.f, 0.f);
      D.ref4[q] = make_float4(0.f, 0.f, 0.f, 0.f);
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
    dp_ligand_order(cx, L, s_perm, s_ltype);
    int end = L;
    for (int a = L - 1; a >= 0; --a) {
      if (a + 1 < L && s_ltype[a + 1] != s_ltype[a]) end = a + 1;
      D.lgrp[a] = make_int2(s_ltype[a], end);
    }
  }
  for (int q = tid; q < nlig * 3; q += blockDim.x) D.lcenter[q] = cx->lig[q / 3].center[q % 3];
  for (int q = tid; q < nprt * 3; q += blockDim.x) D.pcenter[q] = cx->prt[q / 3].pocket_center[q % 3];
  for (int q = tid; q < M; q += blockDim.x) D.tcc[q] = cx->mcs[q].tcc;

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
    s_nk = b;
    if (D.nkde_expect >= 0 && b != D.nkde_expect) dp_fail(D, kPackFailShape, kFieldKde, b);
  }
  __syncthreads();
  for (int t = warp; t < kLigTypes; t += nwarps) {
    int at = s_kbeg[t];
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      const bool m = k < K && cx->kde.t[k] == t;
      const unsigned b = __ballot_sync(0xffffffffu, m);
      if (m && at + __popc(b & ((1u << lane) - 1u)) < D.kde_cap) {
        const int o = at + __popc(b & ((1u << lane) - 1u));
        D.kde[o] = make_float4(cx->kde.x[k], cx->kde.y[k], cx->kde.z[k], dp_as_float(t));
      }
      at += __popc(b);
    }
  }
  if (tid == 0 && s_nk == 0 && D.kde_cap > 0) D.kde[0] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncthreads();
  // KDE slots (the host packer's order): for each ligand type group, each KDE
  // point of its type, with the group's atom range and 1/(points of the type)
  __shared__ int s_ga[kLigTypes], s_ge[kLigTypes], s_gt[kLigTypes], s_go[kLigTypes + 1], s_ng, s_valid;
  // (only for a valid Complex: with an out-of-range ligand type the grouped
  // order does not cover every atom)
  if (tid == 0) s_valid = (*(volatile int *)D.err & kErrPack) == 0;
  __syncthreads();
  if (D.kslot && s_valid) {
    if (tid == 0) {
      int ng = 0, off = 0;
      for (int a = 0; a < L;) {
        const int t = s_ltype[a];
        int e = a;
        while (e < L && s_ltype[e] == t) ++e;
        if (s_kcnt[t] > 0) {
          s_ga[ng] = a;
          s_ge[ng] = e;
          s_gt[ng] = t;
          s_go[ng] = off;
          off += s_kcnt[t];
          ++ng;
        }
        a = e;
      }
      s_go[ng] = off;
      s_ng = ng;
    }
    __syncthreads();
    const int nslot = s_go[s_ng];
    for (int q = tid; q < nslot && q < D.kde_cap; q += blockDim.x) {
      int g = 0;
      while (q >= s_go[g + 1]) ++g;
      const int t = s_gt[g];
      const float4 p = D.kde[s_kbeg[t] + (q - s_go[g])];
      const float inv = 1.0f / (float)s_kcnt[t];
      D.kslot[2 * q] = make_int4(__float_as_int(p.x), __float_as_int(p.y), __float_as_int(p.z), __float_as_int(inv));
      D.kslot[2 * q + 1] = make_int4(s_ga[g] | (s_ge[g] << 16), 0, 0, 0);
    }
    __syncthreads();
  }
  // the header only for a valid Complex: the kernels that read it run only then
  if (tid == 0 && (*(volatile int *)D.err & kErrPack) == 0) {
    DevJob J;
    J.natom = L;
    J.nlig = nlig;
    J.lstride = (L + 3) & ~3;
    J.lig = D.lig;
    J.lgrp = D.lgrp;
    J.lcenter = D.lcenter;
    J.npoint_pad = s_P;
    J.nprt = nprt;
    J.pos = D.pos;
    J.aux = D.aux;
    J.ncdc = D.ncdc;
    J.pcenter = D.pcenter;
    J.psp = D.psp;
    J.pspmask = D.pspmask;
    J.pcell = D.pcell;
    J.pcell_cnt = D.pcell_cnt;
    J.pcell_stride = D.pcell_stride;
    for (int t = 0; t < kLigTypes; ++t) {
      J.kbeg[t] = s_kbeg[t];
      J.kcnt[t] = s_kcnt[t];
    }
    J.nkde = s_nk;
    J.kde = D.kde;
    J.nkslot = (D.kslot && s_valid) ? min(s_go[s_ng], D.kde_cap) : 0;
    J.kslot = D.kslot;
    J.nmcs = M;
    J.mcs = D.mcs;
    J.tcc = D.tcc;
    J.ntmp = D.rep ? s_ntmp : 0;
    J.minus_beta = D.minus_beta;
    J.par = D.par;
    J.ref4 = D.ref4;
    J.nrep = D.rep ? D.nrep : 0;
    J.rep = D.rep;
    J.run_acc = D.run_acc;
    J.stats = D.stats;
    J.rec = D.rec;
    J.key0 = D.key0;
    J.key1 = D.key1;
    J.rid_base = D.rep ? D.rep_begin : 0;
    J.nrep_total = D.rep ? D.nrep_total : 0;
    J.step0 = 0;
    J.nsteps = 0;
    J.xsweep = -1;
    J.pad_ = 0;
    *D.job = J;
  }
}

// One CTA per protein conformation: points ordered as the host packer orders
// them (hydrophobic-contact points first, each part by hydrogen-bond group and point type,
// stable; 60 buckets (cdc, type), two per warp, counted and scattered with
// warp ballots), inert padding, the pocket-specific potential gathered with
// its non-zero type mask, and its non-zero cells for the ligand's types, by
// type then point (one warp per type, counted and scattered the same way).
__global__ void __launch_bounds__(1024) dp_pocket_kernel(const Complex *__restrict__ cx, PackDst D)
{
  constexpr int kBuckets = 2 * kPadType;
  __shared__ int s_cnt[kBuckets], s_beg[kBuckets], s_rank[kPadType];
  if (*(volatile int *)D.err & kErrPack) return;
  const int i = blockIdx.x;
  const int nprt = cx->size.n_prt;
  if (i >= nprt) return;
  const Protein &pr = cx->prt[i];
  int P = 0;
  for (int c = 0; c < nprt; ++c) P = max(P, cx->prt[c].prt_npoint);
  const int np = pr.prt_npoint;
  const int Pp = D.Ppad > 0 ? D.Ppad : ((P + kPointAlign - 1) / kPointAlign) * kPointAlign;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // the host packer's order: per part (cdc == 1 first) the point types with a
  // hydrogen-bond parameter first, each group by type: rank of each type
  if (threadIdx.x == 0) {
    uint32_t m = 0;
    for (int lt = 0; lt < kLigTypes; ++lt)
      for (int pt = 0; pt < kPadType; ++pt)
        if (cx->enepara.hdb0[lt][pt] > 0.1f) m |= 1u << pt;
    int r = 0;
    for (int pt = 0; pt < kPadType; ++pt)
      if ((m >> pt) & 1u) s_rank[pt] = r++;
    for (int pt = 0; pt < kPadType; ++pt)
      if (!((m >> pt) & 1u)) s_rank[pt] = r++;
  }
  __syncthreads();
  auto bucket = [&](int k) { return (pr.cdc[k] == 1 ? 0 : kPadType) + s_rank[pr.t[k]]; };
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
    D.ncdc[i] = nc;
  }
  __syncthreads();
  float4 *pos = D.pos + (size_t)i * Pp;
  float2 *aux = D.aux + (size_t)i * Pp;
  float *psp = D.psp + (size_t)i * kLigTypes * Pp;
  uint32_t *pm = D.pspmask + (size_t)i * Pp;
  for (int bk = warp; bk < kBuckets; bk += nwarps) {
    int at = s_beg[bk];
    for (int k0 = 0; k0 < np; k0 += 32) {
      const int k = k0 + lane;
      const bool m = k < np && bucket(k) == bk;
      const unsigned b = __ballot_sync(0xffffffffu, m);
      if (m) {
        const int j = at + __popc(b & ((1u << lane) - 1u));
        pos[j] = make_float4(pr.x[k], pr.y[k], pr.z[k], pr.ele[k]);
        aux[j] = make_float2(pr.cdc[k] == 1 ? pr.hpp[k] : 0.f, dp_as_float(pr.t[k]));
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
    aux[j] = make_float2(0.f, dp_as_float(kPadType));
    pm[j] = 0u;
    for (int lt = 0; lt < kLigTypes; ++lt) psp[(size_t)lt * Pp + j] = 0.f;
  }
  if (!D.pcell) return;
  // cells: the atoms of type t are [tbeg, tbeg + tcnt) of the type-grouped ligand
  __shared__ int s_tcnt[kLigTypes], s_tbeg[kLigTypes], s_ccnt[kLigTypes], s_cbeg[kLigTypes];
  __syncthreads();  // this CTA's mask writes above are read below
  const int L = cx->lig[0].lig_natom;
  if (warp < kLigTypes) {
    int na = 0;
    for (int a0 = 0; a0 < L; a0 += 32)
      na += __popc(__ballot_sync(0xffffffffu, a0 + lane < L && cx->lig[0].t2[a0 + lane] == warp));
    int nc = 0;
    if (na > 0)
      for (int j0 = 0; j0 < Pp; j0 += 32)
        nc += __popc(__ballot_sync(0xffffffffu, j0 + lane < Pp && ((pm[j0 + lane] >> warp) & 1u)));
    if (lane == 0) {
      s_tcnt[warp] = na;
      s_ccnt[warp] = nc;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // atom ranges in the grouped ligand's type order, cells by type index
    int order[kLigTypes];
    dp_ligand_type_order(cx, order);
    int a = 0, c = 0;
    for (int q = 0; q < kLigTypes; ++q) {
      s_tbeg[order[q]] = a;
      a += s_tcnt[order[q]];
    }
    for (int t = 0; t < kLigTypes; ++t) {
      s_cbeg[t] = c;
      c += s_ccnt[t];
    }
    D.pcell_cnt[i] = min(c, D.pcell_stride);
    if (c > D.pcell_stride) dp_fail(D, kPackFailCapacity, kFieldPcell, c);
  }
  __syncthreads();
  if (warp < kLigTypes && s_tcnt[warp] > 0) {
    int4 *cell = D.pcell + (size_t)i * D.pcell_stride * 2;
    const int t = warp, rng = s_tbeg[t] | ((s_tbeg[t] + s_tcnt[t]) << 16);
    int at = s_cbeg[t];
    for (int j0 = 0; j0 < Pp; j0 += 32) {
      const int j = j0 + lane;
      const bool m = j < Pp && ((pm[j] >> t) & 1u);
      const unsigned b = __ballot_sync(0xffffffffu, m);
      const int o = at + __popc(b & ((1u << lane) - 1u));
      if (m && o < D.pcell_stride) {
        const float4 q = pos[j];
        const int pt = __float_as_int(aux[j].y);
        cell[2 * o] = make_int4(__float_as_int(q.x), __float_as_int(q.y), __float_as_int(q.z),
                                __float_as_int(psp[(size_t)t * Pp + j]));
        cell[2 * o + 1] = make_int4(rng, __float_as_int(D.par->tab4[t][pt].z), t, j);
      }
      at += __popc(b);
    }
  }
}

// Ligand conformations in grouped atom order, MCS templates atom-major; with a
// replica destination also the replica range, accept flags, statistics and
// the temperature ladder.
__global__ void dp_ligand_kernel(const Complex *__restrict__ cx, PackDst D)
{
  __shared__ int s_perm[GD_MAXLIG], s_ltype[GD_MAXLIG];
  if (*(volatile int *)D.err & kErrPack) return;
  const int L = cx->lig[0].lig_natom, M = cx->size.mcs_nrow, nlig = cx->size.n_lig;
  const int ls = (L + 3) & ~3;
  if (threadIdx.x == 0) dp_ligand_order(cx, L, s_perm, s_ltype);
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  for (int q = g; q < nlig * ls; q += stride) {
    const int i = q / ls, a = q % ls;
    if (a < L) {
      const int s = s_perm[a];
      const Ligand &lg = cx->lig[i];
      D.lig[q] = make_float4(lg.x2[s], lg.y2[s], lg.z2[s], cx->lig[0].c2[s]);
    } else {
      D.lig[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  for (int q = g; q < L * M; q += stride) {
    const int a = q / M, m = q % M;
    const int s = s_perm[a];
    const float x = cx->mcs[m].x[s];
    D.mcs[q] = make_float4(x, cx->mcs[m].y[s], cx->mcs[m].z[s], x != GD_MCS_INVALID_COORD ? 1.f : 0.f);
  }
  if (!D.rep) return;
  const int ntmp = cx->size.n_tmp, nprt = cx->size.n_prt;
  for (int t = g; t < ntmp; t += stride) D.minus_beta[t] = cx->temp[t].minus_beta;
  for (int r = g; r < D.nrep; r += stride) {
    ReplicaMC R = cx->replica[D.rep_begin + r];
    if (R.idx_lig < 0 || R.idx_lig >= nlig || R.idx_prt < 0 || R.idx_prt >= nprt || R.idx_tmp < 0 ||
        R.idx_tmp >= ntmp) {
      dp_fail(D, kPackFailInput, kFieldReplica, D.rep_begin + r);
      R.idx_lig = R.idx_prt = R.idx_tmp = 0;  // in range, whatever reads it before the flag is seen
    }
    D.rep[r] = R;
    D.run_acc[r] = R.is_accept;
    RepStats S;
    S.e_sum = S.e_sum2 = S.best_e = 0.0;
    S.n_steps = S.n_accept = S.n_exch_try = S.n_exch_acc = 0;
    for (int i = 0; i < 6; ++i) S.best_mm[i] = 0.f;
    S.best_step = -1;
    S.pad_ = 0;
    D.stats[r] = S;
  }
}

}  // namespace

cudaError_t device_pack(const Complex *d_cx, const PackDst &D, cudaStream_t st)
{
  (void)cudaGetLastError();  // a failure an earlier call already reported is not this launch's
  dp_setup_kernel<<<1, 256, 0, st>>>(d_cx, D);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dp_pocket_kernel<<<GD_MAX_CONF_PRT, 1024, 0, st>>>(d_cx, D);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dp_ligand_kernel<<<64, 256, 0, st>>>(d_cx, D);
  return cudaGetLastError();
}

const char *pack_field_name(int f)
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
    case kFieldNTmp: return "size.n_tmp (temperatures)";
    case kFieldReplica: return "a replica's conformation or temperature index (replica given)";
    case kFieldPcell: return "non-zero pocket-specific cells of a conformation";
    default: return "unknown field";
  }
}

}  // namespace gd
