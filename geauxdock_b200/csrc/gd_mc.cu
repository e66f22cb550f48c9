// gd_mc.cu -- the batched Monte Carlo kernel (one warp per replica), the
// pose-evaluation kernel that shares its energy code, and the replica
// exchange kernels.
//
// Mapping to the hardware.  The reference runs one 1024-thread block per
// replica and synchronises the block six or more times per step
// (src/backend_gpu/kernel_cuda_l1_montecarlo.cu:284-527).  Here one warp owns
// one replica for a whole chunk of steps: the step needs no block barrier,
// only warp shuffles.  A CTA holds R replica-warps that share one protein
// conformation; per work item the CTA stages the force-field parameters (in
// FP64 also the KDE points; when it pays, the conformation itself) into shared
// memory with 1-D bulk (TMA) copies, and its replica-warps read them every
// step.  A persistent grid takes work items from an atomic queue, heaviest
// first.
//
// Pair loop, pass 1 (every term but the hydrophobic contact).  Lane i holds
// pocket points row+i+32j (j < KPL) in registers.  The FP32 ligand sits in
// shared memory as atom pairs, and with KPL even every add, multiply and FMA
// evaluates atoms 2k and 2k+1 against one point as one packed f32x2
// instruction (sm_100).  Per work item the CTA builds from the per-type tables
// one entry per (atom pair, point type) with the two atoms' values interleaved,
// so the loop walks atom pairs with no grouping by atom type; the sparse
// hydrogen-bond term is evaluated only for the atom pairs where some point of
// the row needs it, and the pocket-specific term is walked after the loop over
// the potential's non-zero cells of the conformation.  With KPL = 1 (and in
// FP64) the atoms are walked one type group at a time in scalar arithmetic,
// the pocket-specific term inside that loop.  Pass 2
// (the hydrophobic contact) visits only the rows holding cdc == 1 points, packed
// over atom pairs the same way, and keeps per-atom sums in registers for AB
// atoms at a time.
//
// Arithmetic follows src/backend_gpu/energy_prt_v1.cu:8-174 term by term, in
// rearranged FP32 forms derived in the comments; the special functions use
// the single-instruction PTX approximations (rsqrt/rcp/ex2.approx).  The
// FP32-Kahan variant (the default) adds each row's partial sums of the three
// dense terms into the lane totals with compensated summation and reduces
// across lanes with a compensated butterfly; the FP64 variant evaluates the
// reference's forms in double.
#include <cstdio>
#include <type_traits>

#include "gd_device.cuh"
#include "gd_internal.h"
#include "gd_pack.h"

namespace gd {

namespace {

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kSqrt2PiInvNeg = -0.3989422804014327f;  // -1/sqrt(2 pi), kernel_cuda_l1_montecarlo.cu:14
constexpr double kSqrt2PiInvNegD = -0.39894228040143267794;  // the same in FP64
// bound of the staging waits when the wait_limit option is 0: one second
constexpr uint64_t kWaitLimitNs = 1000000000ull;

__device__ __forceinline__ uint64_t wait_limit_ns(uint32_t us) { return us ? 1000ull * us : kWaitLimitNs; }

template <typename T>
struct alignas(16) V4 {
  T x, y, z, w;
};

// FP32 ligand in shared memory as atom pairs: component k of each float2 is
// atom 2i + k of pair i, so that packed f32x2 arithmetic reads two atoms as one
// register pair.  An odd atom count ends with an inert dummy half.
struct alignas(16) LigPair {
  float2 x, y, z, q;
};
__device__ __forceinline__ V4<float> atom_at(const LigPair *lig, int a)
{
  const float *f = reinterpret_cast<const float *>(lig + (a >> 1)) + (a & 1);
  return V4<float>{f[0], f[2], f[4], f[6]};
}
__device__ __forceinline__ V4<double> atom_at(const V4<double> *lig, int a) { return lig[a]; }

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

}  // namespace

// Bounds checks of the debug build (-DGD_CHECK, libgdock_check.so): every
// instrumented index is compared with the length of its array; one out of
// range records (site, index, length) in g_check once and is replaced by 0,
// so the access stays inside the array and the run goes on.  gd_check_report
// reads the record.  In the product build GD_AT(i, n, site) is the tokens of i.
#ifdef GD_CHECK
static __device__ int g_check[4];
__device__ __forceinline__ long long check_at(long long i, long long n, int site)
{
  if (i >= 0 && i < n) return i;
  if (atomicCAS(&g_check[0], 0, 1) == 0) {
    g_check[1] = site;
    g_check[2] = (int)i;
    g_check[3] = (int)n;
  }
  return 0;
}
#define GD_AT(i, n, site) ::gd::check_at((long long)(i), (long long)(n), (site))
#define GD_CHECK_ARG(...) , __VA_ARGS__
#else
// unparenthesised on purpose: the index expression keeps its own grouping
// (a pointer plus an index sum is then computed as written), so that the
// product build compiles to exactly the code without the checks.  A use
// inside a product or another operator must parenthesise its argument
// (2 * GD_AT((k + m), ...)), or it would expand to 2 * k + m.
#define GD_AT(i, n, site) i
#define GD_CHECK_ARG(...)
#endif
// sites reported by gd_check_report
enum CheckSite { kSiteLig = 1, kSiteApt, kSiteAph, kSiteAhd, kSitePos, kSitePsp, kSiteKde, kSiteMcs, kSiteLgrp,
                 kSiteTcc, kSiteLigConf, kSitePrtConf, kSiteRep, kSiteTmp, kSiteTab = 16 };

// ----------------------------------------------------------- smem layout --
struct SmemLayout {
  uint32_t params, lgrp, pos, aux, kde, apt, aph, ahd, warp0, warp_bytes, lig_bytes, parts, total;
};

// Per-warp partial sums of a replica split over several warps (latency mode):
// the dense terms, then the hydrophobic sum of every atom.
constexpr int kPartTerms = 8;    // vdw, ele, pmf, psp, hdb, kde, mcs, (1 unused)
constexpr uint32_t kPartBytes = 4u * (kPartTerms + kMaxAtoms);

__host__ __device__ inline uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

__host__ __device__ inline SmemLayout smem_layout(int P, int Kst, int lig_slots, int warps, bool fp64,
                                                   int group = 1)
{
  SmemLayout s;
  uint32_t off = 0;
  s.params = off;  // FP64: the whole DevParams; FP32: its scalar prefix
  off = align16(off + (uint32_t)(fp64 ? sizeof(DevParams) : kParamScalarBytes));
  s.lgrp = off;
  off = align16(off + (uint32_t)sizeof(int2) * kMaxAtoms);
  s.pos = off;
  off = align16(off + 16u * (uint32_t)P);
  s.aux = off;
  off = align16(off + 8u * (uint32_t)P);
  s.kde = off;
  off = align16(off + 16u * (uint32_t)Kst);
  // FP32: per (atom pair, point type) tables of the atom-pair pair loop
  const uint32_t npairs = fp64 ? 0u : (uint32_t)(lig_slots + 1) / 2u;
  s.apt = off;
  off = align16(off + 32u * (uint32_t)kTabCols * npairs);
  s.aph = off;
  off = align16(off + 16u * (uint32_t)kTabCols * npairs);
  s.ahd = off;
  off = align16(off + 16u * npairs);
  s.lig_bytes = (uint32_t)lig_slots * (fp64 ? 32u : 16u);  // V4<double> per atom, or LigPair per two atoms
  // per warp: rotated ligand, ReplicaMC state, EnergyScratch (192 B), WarpStats (64 B), and with
  // several warps per replica its partial sums
  s.parts = s.lig_bytes + (uint32_t)sizeof(ReplicaMC) + 192u + 64u;
  s.warp_bytes = align16(s.parts + (group > 1 ? kPartBytes : 0u));
  s.warp0 = off;
  off += s.warp_bytes * (uint32_t)warps;
  s.total = off;
  return s;
}

// warps per replica a launch runs with: pose evaluation and FP64 use one
template <int MODE, int PREC>
__host__ __device__ inline int kernel_group(const KArgs &a)
{
  return (MODE == 1 || PREC == kFP64 || a.group < 1) ? 1 : a.group;
}

// Barrier of the G warps of one replica (named barrier 1 + index of the group).
__device__ __forceinline__ void group_sync(int bar_id, int G)
{
  asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(G * 32) : "memory");
}

// A replica's place in a group of G warps (latency mode): warp `sub` of the
// group takes pair rows sub, sub + G, ... and KDE points likewise; its partial
// sums go to its own part area (gparts + sub * pstride floats) and warp 0 of
// the group combines them in warp order, so that the result depends on G but
// on nothing else.  G = 1 is the plain one-warp-per-replica evaluation.
struct Split {
  int sub, G, bar_id;
  float *gparts;
  uint32_t pstride;
};
struct NoSplit {};  // the one-warp-per-replica instantiation takes no split argument

// ------------------------------------------------------------- energy --
// Energy of ligand conformation ilig at pose mm in protein conformation iprt.
// Called by all 32 lanes of a warp; on return every lane holds e[0..9]
// (normalised terms and total) and raw[0..8] (terms before normalisation).
// Per-warp results of energy_warp (written by lane 0 after the reductions).
struct EnergyScratch {
  double e[10];    // normalised terms and total
  double raw[9];   // terms before the per-atom division and normalisation
  float mm[6];     // pose being evaluated (input)
  float pad_[4];
};
static_assert(sizeof(EnergyScratch) == 192, "EnergyScratch size is part of the smem layout");

// Running sums of the pair terms of one point row.  The electrostatic term
// q_a q_p g(d) is summed per point as q_p * sum_a q_a g(d), one sum per point
// the lane holds, and multiplied by q_p at the end of the row.
template <typename T, int KPL>
struct PairAcc {
  T vdw, pmf, psp, hdb;
  T ele[KPL];
};

// Scalar force-field constants of the pair terms, read once per pose.
struct PairConst {
  float lj0, lj1, lj01, el0, el1, inv_el1, a1, b1, ea, eb, ed2;
  __device__ static PairConst load(const DevParams *p)
  {
    PairConst c;
    c.lj0 = p->lj0; c.lj1 = p->lj1; c.lj01 = p->lj01; c.el0 = p->el0; c.el1 = p->el1; c.inv_el1 = p->inv_el1;
    c.a1 = p->a1; c.b1 = p->b1; c.ea = p->ele_a; c.eb = p->ele_b; c.ed2 = p->ele_d2max;
    return c;
  }
};

// Pair terms of ligand atoms [a, aend) (one type group) against the lane's
// KPL points, energy_prt_v1.cu:56-139 except the hydrophobic contact.  HDB /
// PSP: evaluate the hydrogen-bond / pocket-specific terms (some lane has a
// non-zero parameter).  FP32 uses rearranged forms of the same formulas
// (t4 = (1/p1a, p2a/p1a, pmf0, pmf1), tab4_entry):
//   LJ = (1 - (p2a/p1a) d^3) / (lj0 + lj0 lj1 d^2 + d^9 / p1a)   (divided through by p1),
//   g  = el0 + d^2 (a1 el1^2 + b1 el1^3 d) for el1 d < 1, else r/el1 with r = 1/d,
//   hdb1 exp(-((d - hdb0) hdb1)^2 / 2) = (hdb1 c) 2^-(d hdb1 c - hdb0 hdb1 c)^2 / c
// (t2 = (hdb1 c, -hdb0 hdb1 c)).  FP64 evaluates the reference's forms with
// rf = (p1a, p2a, hdb0, hdb1).
template <int PREC, int KPL, bool HDB, bool PSP, typename T, typename LA>
__device__ __forceinline__ void pair_atoms(const LA *lig, int a, int aend, const T (&px)[KPL],
                                           const T (&py)[KPL], const T (&pz)[KPL], const float4 (&t4)[KPL],
                                           const float2 (&t2)[KPL], const float4 (&rf)[KPL], const T (&tps)[KPL],
                                           const PairConst &c, PairAcc<T, KPL> &acc)
{
  if constexpr (PREC == kFP64) {
    const double lj0 = c.lj0, lj1 = c.lj1, el0 = c.el0, el1 = c.el1, a1 = c.a1, b1 = c.b1;
    for (; a < aend; ++a) {
      const V4<double> la = atom_at(lig, a);
#pragma unroll
      for (int j = 0; j < KPL; ++j) {
        const double dx = la.x - px[j], dy = la.y - py[j], dz = la.z - pz[j];
        const double d2 = dx * dx + dy * dy + dz * dz;
        const double d4 = d2 * d2;
        const double d = sqrt(d2);
        const double p1 = (double)rf[j].x / (d4 * d4 * d);
        const double p2 = (double)rf[j].y / (d4 * d2);
        const double p4 = p1 * lj0 * (1.0 + lj1 * d2) + 1.0;
        acc.vdw += (p1 - p2) / p4;
        const double s1 = el1 * d;
        const double g = (s1 < 1.0) ? el0 + a1 * s1 * s1 + b1 * s1 * s1 * s1 : 1.0 / s1;
        acc.ele[j] += la.w * g;
        const double dmp = d + (double)t4[j].z;   // t4.z = -pmf0
        acc.pmf += (double)t4[j].w / (1.0 + exp((-0.5 * d + 6.0) * dmp));
        if constexpr (PSP) acc.psp += (dmp <= 0.0) ? tps[j] : 0.0;
        if constexpr (HDB) {
          const double h3 = (d - (double)rf[j].z) * (double)rf[j].w;
          acc.hdb += (double)rf[j].w * exp(-0.5 * h3 * h3);
        }
      }
    }
  } else {
#pragma unroll 2
    for (; a < aend; ++a) {
      const V4<float> la = atom_at(lig, a);
#pragma unroll
      for (int j = 0; j < KPL; ++j) {
        const float dx = la.x - px[j], dy = la.y - py[j], dz = la.z - pz[j];
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float r = rsqrt_approx(d2);
        const float d = d2 * r;
        const float d3 = d2 * d;
        const float d6 = d3 * d3;
        const float den = fmaf(d6 * d3, t4[j].x, fmaf(c.lj01, d2, c.lj0));
        const float num = fmaf(t4[j].y, d3, 1.0f);
        acc.vdw = fmaf(num, rcp_approx(den), acc.vdw);
        const float g = (d2 < c.ed2) ? fmaf(d2, fmaf(c.eb, d, c.ea), c.el0) : r * c.inv_el1;
        acc.ele[j] = fmaf(la.w, g, acc.ele[j]);
        const float dmp = d + t4[j].z;
        const float ex = ex2_approx(fmaf(-0.5f * kLog2e, d, 6.0f * kLog2e) * dmp);
        acc.pmf = fmaf(t4[j].w, rcp_approx(1.0f + ex), acc.pmf);
        if constexpr (PSP) acc.psp += (dmp <= 0.0f) ? tps[j] : 0.0f;
        if constexpr (HDB) {
          const float h = fmaf(d, t2[j].x, t2[j].y);
          acc.hdb = fmaf(t2[j].x, ex2_approx(-(h * h)), acc.hdb);
        }
      }
    }
  }
}

// Running sums of one point row in the atom-pair form: component k of each
// float2 belongs to atom 2i + k of the pair being visited; the electrostatic
// sums are kept per point (they are multiplied by the point charge at the end
// of the row).
template <int KPL>
struct PairAccP {
  float2 vdw, pmf, hdb;
  float2 ele[KPL];
};

// Per work item, shared-memory tables of the atom-pair pair loop, built from
// the per-type tables (read from global memory): for pair i (atoms a = 2i,
// b = 2i + 1) and point type pt, e = i * kTabCols + pt,
//   apt[2e]     = (1/p1a, -p2a/p1a) of a and b interleaved: (a.x, b.x, a.y, b.y)
//   apt[2e + 1] = (-pmf0, pmf1) interleaved
//   aph[e]      = (hdb1 c, -hdb0 hdb1 c) interleaved
//   ahd[i]      = (point types with hydrogen-bond parameters for a or b,
//                  bit set of the types of a and b, type of a, type of b or 31).
// The dummy half of an odd atom count gets the padding column and no types:
// every term of it is exactly 0.
__device__ void build_pair_tables(int L, const DevParams *par, const int2 *lg, float4 *apt, float4 *aph, int4 *ahd)
{
  const int npairs = (L + 1) >> 1;
  for (int e = threadIdx.x; e < npairs * kTabCols; e += blockDim.x) {
    const int i = e / kTabCols, pt = e % kTabCols;
    const int a = 2 * i, b = a + 1;
    const int lta = GD_AT(lg[GD_AT(a, L, kSiteLgrp)].x, kLigTypes, kSiteTab), ltb = b < L ? lg[b].x : -1;
    const float4 ta = par->tab4[lta][pt];
    const float4 tb = ltb >= 0 ? par->tab4[ltb][pt] : tab4_padding();
    apt[2 * e] = make_float4(ta.x, tb.x, ta.y, tb.y);
    apt[2 * e + 1] = make_float4(ta.z, tb.z, ta.w, tb.w);
    const float2 ha = par->tab2[lta][pt], hb = ltb >= 0 ? par->tab2[ltb][pt] : make_float2(0.f, 0.f);
    aph[e] = make_float4(ha.x, hb.x, ha.y, hb.y);
    if (pt == 0) {
      const uint32_t hm = par->hdbmask[lta] | (ltb >= 0 ? par->hdbmask[ltb] : 0u);
      const uint32_t tb_bits = (1u << lta) | (ltb >= 0 ? 1u << ltb : 0u);
      ahd[i] = make_int4((int)hm, (int)tb_bits, lta, ltb >= 0 ? ltb : 31);
    }
  }
}

// Pair terms of ligand atom pair i against the lane's KPL points
// (energy_prt_v1.cu:56-139 except the hydrophobic contact), the FP32 forms of
// pair_atoms with two atoms per packed f32x2 instruction (__ffma2_rn /
// __fadd2_rn / __fmul2_rn, sm_100); the special functions stay per component.
// HDB: evaluate the hydrogen-bond term (some point of the row has a parameter
// for one of the two atoms); the pocket-specific term is walked over its
// non-zero cells after the loop.  npx/npy/npz hold the lane's negated point
// coordinates twice (x_atom - x_point is x_atom + (-x_point), exactly); the
// charges are read from shared memory where they are used, which keeps the
// loop within its registers.
template <int KPL, bool HDB>
__device__ __forceinline__ void pair_atom_pair(const LigPair *__restrict__ lig, int i GD_CHECK_ARG(int npairs), const float2 &lx,
                                               const float2 &ly, const float2 &lz, const float4 *__restrict__ apt,
                                               const float4 *__restrict__ aph, const int (&pt)[KPL],
                                               const float2 (&npx)[KPL], const float2 (&npy)[KPL],
                                               const float2 (&npz)[KPL], const PairConst &c, PairAccP<KPL> &acc)
{
  const float2 lj01 = f2(c.lj01), lj0 = f2(c.lj0), one = f2(1.0f), inv_el1 = f2(c.inv_el1);
  const float2 za = f2(-0.5f * kLog2e), zb = f2(6.0f * kLog2e);
#pragma unroll
  for (int j = 0; j < KPL; ++j) {
    const int e = i * kTabCols + pt[j];
    const float4 ta = apt[2 * e], tb = apt[GD_AT(2 * e + 1, 2 * npairs * kTabCols, kSiteApt)];
    const float2 dx = __fadd2_rn(lx, npx[j]), dy = __fadd2_rn(ly, npy[j]), dz = __fadd2_rn(lz, npz[j]);
    const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    const float2 r = make_float2(rsqrt_approx(d2.x), rsqrt_approx(d2.y));
    const float2 d = __fmul2_rn(d2, r);
    const float2 d3 = __fmul2_rn(d2, d);
    const float2 d6 = __fmul2_rn(d3, d3);
    const float2 den = __ffma2_rn(__fmul2_rn(d6, d3), make_float2(ta.x, ta.y), __ffma2_rn(lj01, d2, lj0));
    const float2 num = __ffma2_rn(make_float2(ta.z, ta.w), d3, one);
    acc.vdw = __ffma2_rn(num, make_float2(rcp_approx(den.x), rcp_approx(den.y)), acc.vdw);
    float2 g = __fmul2_rn(r, inv_el1);
    if (d2.x < c.ed2) g.x = fmaf(d2.x, fmaf(c.eb, d.x, c.ea), c.el0);
    if (d2.y < c.ed2) g.y = fmaf(d2.y, fmaf(c.eb, d.y, c.ea), c.el0);
    acc.ele[j] = __ffma2_rn(lig[GD_AT(i, npairs, kSiteLig)].q, g, acc.ele[j]);
    const float2 dmp = __fadd2_rn(d, make_float2(tb.x, tb.y));
    const float2 z = __fmul2_rn(__ffma2_rn(za, d, zb), dmp);
    const float2 e1 = __fadd2_rn(make_float2(ex2_approx(z.x), ex2_approx(z.y)), one);
    acc.pmf = __ffma2_rn(make_float2(tb.z, tb.w), make_float2(rcp_approx(e1.x), rcp_approx(e1.y)), acc.pmf);
    if constexpr (HDB) {
      const float4 th = aph[GD_AT(e, npairs * kTabCols, kSiteAph)];
      const float2 h = __ffma2_rn(d, make_float2(th.x, th.y), make_float2(th.z, th.w));
      const float2 hh = __fmul2_rn(h, h);
      acc.hdb = __ffma2_rn(make_float2(th.x, th.y), make_float2(ex2_approx(-hh.x), ex2_approx(-hh.y)), acc.hdb);
    }
  }
}

template <int PREC, int KPL, int AB, bool SPLIT = false>
__device__ __noinline__ void energy_warp(const DevJob &J, const DevParams *__restrict__ par,
                                         const float4 *__restrict__ pos, const float2 *__restrict__ aux,
                                         const float4 *__restrict__ kde, const int2 *__restrict__ lgrp,
                                         const float4 *__restrict__ apt, const float4 *__restrict__ aph,
                                         const int4 *__restrict__ ahd, void *ligbuf, int ilig, int iprt,
                                         const float *mm, EnergyScratch *out,
                                         typename std::conditional<SPLIT, Split, NoSplit>::type sp = {})
{
  using T = typename std::conditional<PREC == kFP64, double, float>::type;
  // SPLIT: the latency-mode instantiation (G warps per replica); otherwise G is 1 at compile time
  int G = 1, my_sub = 0;
  if constexpr (SPLIT && PREC != kFP64) {
    G = sp.G;
    my_sub = sp.sub;
  }
  const int row0 = 32 * KPL * my_sub, rstep = 32 * KPL * G;
  const int lane = lane_id();
  const int L = J.natom;
  const int P = J.npoint_pad;
  using LA = typename std::conditional<PREC == kFP64, V4<double>, LigPair>::type;
  LA *lig = reinterpret_cast<LA *>(ligbuf);

  // rotation + translation, kernel_cuda_l1_montecarlo.cu:336-380
  T r00, r01, r02, r10, r11, r12, r20, r21, r22;
  {
    T s1, c1, s2, c2, s3, c3;
    if constexpr (PREC == kFP64) {
      sincos((double)mm[3], &s1, &c1);
      sincos((double)mm[4], &s2, &c2);
      sincos((double)mm[5], &s3, &c3);
    } else {
      sincosf(mm[3], &s1, &c1);
      sincosf(mm[4], &s2, &c2);
      sincosf(mm[5], &s3, &c3);
    }
    r00 = c1 * c2;
    r01 = c1 * s2 * s3 - c3 * s1;
    r02 = s1 * s3 + c1 * c3 * s2;
    r10 = c2 * s1;
    r11 = c1 * c3 + s1 * s2 * s3;
    r12 = c3 * s1 * s2 - c1 * s3;
    r20 = -s2;
    r21 = c2 * s3;
    r22 = c2 * c3;
  }
  const float *lc = J.lcenter + 3 * GD_AT(ilig, J.nlig, kSiteLigConf);
  const T tx = (T)mm[0] + (T)lc[0], ty = (T)mm[1] + (T)lc[1], tz = (T)mm[2] + (T)lc[2];
  const float4 *lsrc = J.lig + (size_t)ilig * J.lstride;
  for (int a = lane; a < L; a += 32) {
    const float4 v = lsrc[a];
    V4<T> o;
    o.x = r00 * (T)v.x + r01 * (T)v.y + r02 * (T)v.z + tx;
    o.y = r10 * (T)v.x + r11 * (T)v.y + r12 * (T)v.z + ty;
    o.z = r20 * (T)v.x + r21 * (T)v.y + r22 * (T)v.z + tz;
    o.w = (T)v.w;
    if constexpr (PREC == kFP64) {
      lig[a] = o;
    } else {
      float *f = reinterpret_cast<float *>(lig + (a >> 1)) + (a & 1);
      f[0] = o.x;
      f[2] = o.y;
      f[4] = o.z;
      f[6] = o.w;
    }
  }
  if constexpr (PREC != kFP64) {
    // the dummy half of an odd atom count: far from every point (padding
    // points sit near +1e4), no charge; its table entries make every term 0
    if ((L & 1) && lane == 0) {
      float *f = reinterpret_cast<float *>(lig + (L >> 1)) + 1;
      f[0] = -1.0e4f;
      f[2] = -1.0e4f;
      f[4] = -1.0e4f;
      f[6] = 0.0f;
    }
  }
  __syncwarp();

  // ---- protein-ligand pair terms, energy_prt_v1.cu:8-174
  // Pass 1: every term but the hydrophobic contact.  Lane i holds points
  // row + i + 32 j (j < KPL); atoms are visited one type group at a time, with
  // the (atom type, point type) table entries loaded once per group.  The
  // hydrogen-bond and pocket-specific terms are skipped for a group when no
  // lane of the warp has a non-zero parameter for it (both are sparse).
  T s_vdw = 0, s_ele = 0, s_pmf = 0, s_psp = 0, s_hdb = 0;
  // Kahan compensations of the three dense sums (psp and hdb are short, sparse sums)
  float c_vdw = 0.f, c_ele = 0.f, c_pmf = 0.f;
  const float *pspc = J.psp + (size_t)iprt * kLigTypes * P;
  const uint32_t *pmc = J.pspmask + (size_t)iprt * P;
  const PairConst kc = PairConst::load(par);

  if constexpr (PREC != kFP64 && KPL % 2 == 0) {
    // atom-pair form: atoms 2i and 2i+1 share one register pair and the
    // table entries come per atom pair, so there is no loop over type groups
    // (the pocket-specific term is not in this loop: it walks the potential's
    // non-zero cells after it)
    const LigPair *lp = lig;
    const int npairs = (L + 1) >> 1;
    for (int row = row0; row < P; row += rstep) {
      float2 npx[KPL], npy[KPL], npz[KPL];
      int pt[KPL];
      uint32_t ptbits = 0u;
#pragma unroll
      for (int j = 0; j < KPL; ++j) {
        const int p = GD_AT(row + 32 * j + lane, P, kSitePos);
        const float4 q = pos[p];
        npx[j] = f2(-q.x);
        npy[j] = f2(-q.y);
        npz[j] = f2(-q.z);
        pt[j] = __float_as_int(aux[p].y);
        ptbits |= 1u << pt[j];
      }
      // point types present in the row: decide per atom pair, for the whole
      // warp, whether the hydrogen-bond term is evaluated
      ptbits = __reduce_or_sync(0xffffffffu, ptbits);
      PairAccP<KPL> acc;
      acc.vdw = acc.pmf = acc.hdb = f2(0.0f);
#pragma unroll
      for (int j = 0; j < KPL; ++j) acc.ele[j] = f2(0.0f);
      for (int i = 0; i < npairs; ++i) {
        const int2 fl = *reinterpret_cast<const int2 *>(&ahd[GD_AT(i, npairs, kSiteAhd)].x);
        const bool any_hdb = ((uint32_t)fl.x & ptbits) != 0u;
        const float4 l01 = *reinterpret_cast<const float4 *>(&lp[GD_AT(i, npairs, kSiteLig)].x);
        const float2 lx = make_float2(l01.x, l01.y), ly = make_float2(l01.z, l01.w), lz = lp[i].z;
        if (any_hdb)
          pair_atom_pair<KPL, true>(lp, i GD_CHECK_ARG(npairs), lx, ly, lz, apt, aph, pt, npx, npy, npz, kc, acc);
        else
          pair_atom_pair<KPL, false>(lp, i GD_CHECK_ARG(npairs), lx, ly, lz, apt, aph, pt, npx, npy, npz, kc, acc);
      }
      float row_ele = 0.f;
#pragma unroll
      for (int j = 0; j < KPL; ++j) {
        // the point charges are read again here rather than held through the atom loop
        row_ele += pos[row + 32 * j + lane].w * (acc.ele[j].x + acc.ele[j].y);
      }
      const float row_vdw = acc.vdw.x + acc.vdw.y, row_pmf = acc.pmf.x + acc.pmf.y;
      const float row_hdb = acc.hdb.x + acc.hdb.y;
      if constexpr (PREC == kFP32Kahan) {
        kahan_add(s_vdw, c_vdw, row_vdw);
        kahan_add(s_ele, c_ele, row_ele);
        kahan_add(s_pmf, c_pmf, row_pmf);
        s_hdb += row_hdb;
      } else {
        s_vdw += row_vdw;
        s_ele += row_ele;
        s_pmf += row_pmf;
        s_hdb += row_hdb;
      }
    }
    // Pocket-specific term (energy_prt_v1.cu:109-115) over the conformation's
    // non-zero cells (point p, ligand type t, value v; only types the ligand
    // has), ordered by type: lane k takes cell k and counts the atoms of type t
    // (the contiguous range [beg, end) of the type-grouped ligand) with
    // d - pmf0 <= 0.  d, -pmf0 (the value the pair tables hold) and the
    // comparison are the pair loop's operations in the same order, so an atom
    // counts here exactly where that loop would count it.
    {
      const int4 *cell = J.pcell + (size_t)iprt * J.pcell_stride * 2;
      const int ncell = J.pcell_cnt[iprt];
      float acc_psp = 0.0f;
      for (int k = 32 * my_sub + lane; k < ncell; k += 32 * G) {
        // the point's coordinates and value, and the atom range with -pmf0 of
        // (t, point type), the pair table's value: two independent 16-byte loads
        const int4 c0 = __ldg(cell + 2 * GD_AT(k, J.pcell_stride, kSitePsp));
        const int4 c1 = __ldg(cell + 2 * k + 1);
        const int beg = c1.x & 0xffff, end = c1.x >> 16;
        const float thr = __int_as_float(c1.y);
        const float nx = -__int_as_float(c0.x), ny = -__int_as_float(c0.y), nz = -__int_as_float(c0.z);
        int hits = 0;
        for (int a = beg; a < end; ++a) {
          const V4<float> la = atom_at(lp, GD_AT(a, L, kSiteLig));
          const float dx = __fadd_rn(la.x, nx), dy = __fadd_rn(la.y, ny), dz = __fadd_rn(la.z, nz);
          const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
          const float d = __fmul_rn(d2, rsqrt_approx(d2));
          hits += __fadd_rn(d, thr) <= 0.0f ? 1 : 0;
        }
        acc_psp = fmaf((float)hits, __int_as_float(c0.w), acc_psp);
      }
      s_psp += acc_psp;
    }
  } else {
    for (int row = row0; row < P; row += rstep) {
      T px[KPL], py[KPL], pz[KPL], pe[KPL];
      int pt[KPL];
      uint32_t pm[KPL];
      uint32_t ptbits = 0u, pmbits = 0u;
  #pragma unroll
      for (int j = 0; j < KPL; ++j) {
        const int p = GD_AT(row + 32 * j + lane, P, kSitePos);
        const float4 q = pos[p];
        px[j] = q.x; py[j] = q.y; pz[j] = q.z; pe[j] = q.w;
        pt[j] = __float_as_int(aux[p].y);
        pm[j] = __ldg(pmc + p);
        ptbits |= 1u << pt[j];
        pmbits |= pm[j];
      }
      // point types present in the row, and ligand types with a pocket-specific
      // potential on some point of it: decide per type group, for the whole warp,
      // whether the sparse terms are evaluated
      ptbits = __reduce_or_sync(0xffffffffu, ptbits);
      pmbits = __reduce_or_sync(0xffffffffu, pmbits);
      PairAcc<T, KPL> acc;
      acc.vdw = acc.pmf = acc.psp = acc.hdb = 0;
  #pragma unroll
      for (int j = 0; j < KPL; ++j) acc.ele[j] = 0;
      int a = 0;
      while (a < L) {
        const int2 grp = lgrp[GD_AT(a, L, kSiteLgrp)];
        const int lt = GD_AT(grp.x, kLigTypes, kSiteTab), aend = grp.y;
        const bool any_hdb = (par->hdbmask[lt] & ptbits) != 0u;
        const bool any_psp = ((pmbits >> lt) & 1u) != 0u;
        float4 t4[KPL], rf[KPL];
        float2 t2[KPL];
        T tps[KPL];
  #pragma unroll
        for (int j = 0; j < KPL; ++j) {
          t4[j] = (PREC == kFP64 ? par : J.par)->tab4[lt][pt[j]];  // FP32 stages no tables
          if constexpr (PREC == kFP64) rf[j] = __ldg(J.ref4 + lt * kTabCols + pt[j]);
          else rf[j] = make_float4(0.f, 0.f, 0.f, 0.f);
          t2[j] = make_float2(0.f, 0.f);
          tps[j] = 0;
        }
        if constexpr (PREC != kFP64) {
          if (any_hdb) {
  #pragma unroll
            for (int j = 0; j < KPL; ++j) t2[j] = J.par->tab2[lt][pt[j]];
          }
        }
        if (any_psp) {
  #pragma unroll
          for (int j = 0; j < KPL; ++j)
            if ((pm[j] >> lt) & 1u) tps[j] = __ldg(pspc + GD_AT((size_t)lt * P + row + 32 * j + lane, kLigTypes * P, kSitePsp));
        }
        if (any_hdb) {
          if (any_psp) pair_atoms<PREC, KPL, true, true>(lig, a, aend, px, py, pz, t4, t2, rf, tps, kc, acc);
          else pair_atoms<PREC, KPL, true, false>(lig, a, aend, px, py, pz, t4, t2, rf, tps, kc, acc);
        } else {
          if (any_psp) pair_atoms<PREC, KPL, false, true>(lig, a, aend, px, py, pz, t4, t2, rf, tps, kc, acc);
          else pair_atoms<PREC, KPL, false, false>(lig, a, aend, px, py, pz, t4, t2, rf, tps, kc, acc);
        }
        a = aend;
      }
      T row_ele = 0;
  #pragma unroll
      for (int j = 0; j < KPL; ++j) row_ele += pe[j] * acc.ele[j];
      if constexpr (PREC == kFP32Kahan) {
        kahan_add(s_vdw, c_vdw, acc.vdw);
        kahan_add(s_ele, c_ele, row_ele);
        kahan_add(s_pmf, c_pmf, acc.pmf);
        s_psp += acc.psp;
        s_hdb += acc.hdb;
      } else {
        s_vdw += acc.vdw;
        s_ele += row_ele;
        s_pmf += acc.pmf;
        s_psp += acc.psp;
        s_hdb += acc.hdb;
      }
    }
  }

  // Pass 2: hydrophobic contact (energy_prt_v1.cu:42-49) over the rows that
  // hold cdc == 1 points (placed first).  The polynomial
  // 1 - 3.5x + 4.5x^2 - 2.5x^3 + 0.5x^4 (x = d^2/81) is (1-x)^3 (1-x/2), i.e.
  // (y^3 + y^4) / 2 with y = 1 - x; clamping y at 0 applies the d^2 <= 81
  // cut-off.  Per-atom sums stay in
  // registers for AB atoms at a time, then the per-atom restraint
  // (energy_prt_v1.cu:162-169).
  T ehpc = 0;
  {
    const int rows = ((J.ncdc[iprt] + 32 * KPL - 1) / (32 * KPL)) * (32 * KPL);
    for (int a0 = 0; a0 < L; a0 += AB) {
      T hpc[AB];
      if constexpr (PREC != kFP64 && KPL % 2 == 0) {
        // atom-pair form, the same operations per component: h2[k] holds the
        // sums of atoms a0 + 2k and a0 + 2k + 1 (AB is even) of hpp (y^2 (y + y^2)),
        // twice the contact sum (halved exactly at the end)
        const float2 one = f2(1.0f), c1 = f2(-1.0f / 81.0f);
        // rows of at most 64 points here: the last row of the hydrophobic-contact
        // points then carries at most 63 others (hpp 0) where 128-point rows
        // would carry up to 127
        constexpr int K2 = KPL > 2 ? 2 : KPL;
        const int rows2 = ((J.ncdc[iprt] + 32 * K2 - 1) / (32 * K2)) * (32 * K2);
        float2 h2[AB / 2];
#pragma unroll
        for (int k = 0; k < AB / 2; ++k) h2[k] = f2(0.0f);
        for (int row = 32 * K2 * my_sub; row < rows2; row += 32 * K2 * G) {
          float2 npx[K2], npy[K2], npz[K2], ph2[K2];
#pragma unroll
          for (int j = 0; j < K2; ++j) {
            const int p = GD_AT(row + 32 * j + lane, P, kSitePos);
            const float4 q = pos[p];
            npx[j] = f2(-q.x);
            npy[j] = f2(-q.y);
            npz[j] = f2(-q.z);
            ph2[j] = f2(aux[p].x);
          }
#pragma unroll
          for (int k = 0; k < AB / 2; ++k) {
            const int a = a0 + 2 * k;
            if (a >= L) break;
            const LigPair la = lig[GD_AT(a >> 1, (L + 1) >> 1, kSiteLig)];
#pragma unroll
            for (int j = 0; j < K2; ++j) {
              const float2 dx = __fadd2_rn(la.x, npx[j]), dy = __fadd2_rn(la.y, npy[j]), dz = __fadd2_rn(la.z, npz[j]);
              const float2 d2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
              float2 y = __ffma2_rn(d2, c1, one);
              y.x = fmaxf(y.x, 0.0f);
              y.y = fmaxf(y.y, 0.0f);
              const float2 yy = __fmul2_rn(y, y);
              const float2 w = __fmul2_rn(yy, __fadd2_rn(y, yy));
              h2[k] = __ffma2_rn(ph2[j], w, h2[k]);
            }
          }
        }
#pragma unroll
        for (int k = 0; k < AB / 2; ++k) {
          hpc[2 * k] = 0.5f * h2[k].x;
          hpc[2 * k + 1] = 0.5f * h2[k].y;
        }
      } else {
#pragma unroll
        for (int k = 0; k < AB; ++k) hpc[k] = 0;
        for (int row = row0; row < rows; row += rstep) {
          T px[KPL], py[KPL], pz[KPL], ph[KPL];
#pragma unroll
          for (int j = 0; j < KPL; ++j) {
            const int p = GD_AT(row + 32 * j + lane, P, kSitePos);
            const float4 q = pos[p];
            px[j] = q.x; py[j] = q.y; pz[j] = q.z;
            ph[j] = aux[p].x;
          }
#pragma unroll
          for (int k = 0; k < AB; ++k) {
            const int a = a0 + k;
            if (a >= L) break;
            const V4<T> la = atom_at(lig, a);
#pragma unroll
            for (int j = 0; j < KPL; ++j) {
              const T dx = la.x - px[j], dy = la.y - py[j], dz = la.z - pz[j];
              const T d2 = dx * dx + dy * dy + dz * dz;
              T t, u;
              if constexpr (PREC == kFP64) {
                t = fmax(1.0 - d2 / 81.0, 0.0);
                u = 1.0 - 0.5 * d2 / 81.0;
              } else {
                t = fmaxf(fmaf(d2, -1.0f / 81.0f, 1.0f), 0.0f);
                u = fmaf(d2, -0.5f / 81.0f, 1.0f);
              }
              hpc[k] += ph[j] * (t * t * t * u);
            }
          }
        }
      }
      if constexpr (PREC != kFP64 && KPL % 2 == 0) {
        // the block's AB contact sums reduced across the warp together: each
        // butterfly step halves the sums a lane carries (it keeps the half its
        // lane bit selects and adds its partner's copy of it), then plain steps
        // finish; lane l ends with atom a0 + base's sum, as do the lanes that
        // differ from it below bit log2(32 / AB).  One lane per atom applies the
        // restraint; its per-lane terms are summed once after the last block.
        float v[AB];
#pragma unroll
        for (int k = 0; k < AB; ++k) v[k] = hpc[k];
        int base = 0;
#pragma unroll
        for (int n = AB, off = 16; n > 1; n >>= 1, off >>= 1) {
          const bool hi = (lane & off) != 0;
#pragma unroll
          for (int i = 0; i < n / 2; ++i) {
            const float keep = hi ? v[n / 2 + i] : v[i], give = hi ? v[i] : v[n / 2 + i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, give, off);
          }
          base += hi ? n / 2 : 0;
        }
#pragma unroll
        for (int off = 16 / AB; off > 0; off >>= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], off);
        const int a = a0 + base;
        if (a < L && (lane & (32 / AB - 1)) == 0) {
          bool restraint = true;
          if constexpr (SPLIT) {
            if (G > 1) {
              // this warp's share of atom a's contact sum; the restraint comes after the combination
              sp.gparts[sp.sub * sp.pstride + kPartTerms + a] = v[0];
              restraint = false;
            }
          }
          if (restraint) {
            const int lt = GD_AT(lgrp[GD_AT(a, L, kSiteLgrp)].x, kLigTypes, kSiteTab);
            const float h2 = (v[0] - par->hpl0[lt]) / par->hpl1[lt];
            ehpc += 0.5f * h2 * h2 - par->hpl2[lt];
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < AB; ++k) {
          const int a = a0 + k;
          if (a >= L) break;
          const T S = warp_sum(hpc[k]);
          const int lt = GD_AT(lgrp[GD_AT(a, L, kSiteLgrp)].x, kLigTypes, kSiteTab);
          const T h2 = (S - (T)par->hpl0[lt]) / (T)par->hpl1[lt];
          ehpc += (T)0.5 * h2 * h2 - (T)par->hpl2[lt];
        }
      }
    }
    // the atom-pair form's restraint terms sit on one lane per atom
    if constexpr (PREC != kFP64 && KPL % 2 == 0) ehpc = warp_sum(ehpc);
  }

  T vdw, ele, pmf, psp, hdb;
  if constexpr (PREC == kFP32Kahan) {
    vdw = warp_sum_comp(s_vdw, c_vdw);
    ele = warp_sum_comp(s_ele, c_ele);
    pmf = warp_sum_comp(s_pmf, c_pmf);
    psp = warp_sum(s_psp);
    hdb = warp_sum(s_hdb);
  } else {
    vdw = warp_sum(s_vdw);
    ele = warp_sum(s_ele);
    pmf = warp_sum(s_pmf);
    psp = warp_sum(s_psp);
    hdb = warp_sum(s_hdb);
  }
  // the FP32 hydrogen-bond sum carries the table's factor c (see DevParams)
  if constexpr (PREC != kFP64) hdb *= par->hdb_cinv;

  // ---- KDE, energy_kde_v1.cu:183-274: per atom, mean of exp(kde2 d^2) over
  // the KDE points of the same type; atoms with no such point contribute 0.
  // The atom-pair form walks the job's slots (below); the per-type-group form:
  // one type group at a time, lane k holds KDE point k of the group's type and
  // sums over the group's atoms, then scales by 1 / (points of the type).  A
  // replica split over G warps deals the slots or the type groups out to its
  // warps in turn.
  T kacc = 0;
  if constexpr (PREC != kFP64 && KPL % 2 == 0) {
    // the atom-pair form walks the job's KDE slots: lane k takes slot k (one
    // KDE point of one of the ligand's type groups) and sums over the group's
    // atoms, weighted by 1/(points of the type): every lane busy, one
    // coalesced pair of loads per slot, no division
    const float k2 = par->kde2 * kLog2e;
    for (int q = 32 * my_sub + lane; q < J.nkslot; q += 32 * G) {
      const int4 c0 = __ldg(J.kslot + 2 * GD_AT(q, J.nkde, kSiteKde));
      const int4 c1 = __ldg(J.kslot + 2 * q + 1);
      const float qx = __int_as_float(c0.x), qy = __int_as_float(c0.y), qz = __int_as_float(c0.z);
      float sk = 0.0f;
      const int end = c1.x >> 16;
      for (int b = c1.x & 0xffff; b < end; ++b) {
        const V4<float> la = atom_at(lig, GD_AT(b, L, kSiteLig));
        const float dx = la.x - qx, dy = la.y - qy, dz = la.z - qz;
        const float d2 = dx * dx + dy * dy + dz * dz;
        sk += ex2_approx(k2 * d2);
      }
      kacc += sk * __int_as_float(c0.w);
    }
  } else {
    const T kde2 = par->kde2;
    int tg = 0;
    for (int a = 0; a < L; ++tg) {
      const int2 grp = lgrp[GD_AT(a, L, kSiteLgrp)];
      const int lt = GD_AT(grp.x, kLigTypes, kSiteTab), aend = grp.y;
      const int cnt = J.kcnt[lt];
      if (cnt > 0 && (G == 1 || tg % G == my_sub)) {
        const int beg = J.kbeg[lt];
        const T inv = (T)1 / (T)cnt;
        for (int k = beg + lane; k < beg + cnt; k += 32) {
          const float4 q = kde[GD_AT(k, J.nkde, kSiteKde)];
          T s = 0;
          for (int b = a; b < aend; ++b) {
            const V4<T> la = atom_at(lig, b);
            const T dx = la.x - (T)q.x, dy = la.y - (T)q.y, dz = la.z - (T)q.z;
            const T d2 = dx * dx + dy * dy + dz * dz;
            if constexpr (PREC == kFP64) s += exp(kde2 * d2);
            else s += ex2_approx((kde2 * kLog2e) * d2);
          }
          kacc += s * inv;
        }
      }
      a = aend;
    }
  }
  T ekde;
  if constexpr (PREC == kFP64) ekde = warp_sum(kacc) / (double)par->kde3;
  else ekde = warp_sum(kacc) * par->kde3_inv;


  // ---- MCS, energy_mcs_v1.cu:277-320
  T macc = 0;
  {
    const int M = J.nmcs;
    if (M <= 16) {
      // two half-warps share each template: lane and lane + 16 take its even and odd atoms
      const int m = lane & 15, h = lane >> 4;
      T s = 0;
      int n = 0;
      // a replica split over G warps deals the templates out to its warps
      const bool mine = m < M && (G == 1 || m % G == my_sub);
      if (mine) {
        for (int a = h; a < L; a += 2) {
          const float4 q = J.mcs[GD_AT((size_t)a * M + m, (size_t)L * M, kSiteMcs)];
          if (q.w != 0.0f) {
            const V4<T> la = atom_at(lig, a);
            const T dx = la.x - (T)q.x, dy = la.y - (T)q.y, dz = la.z - (T)q.z;
            s += dx * dx + dy * dy + dz * dz;
            ++n;
          }
        }
      }
      s += __shfl_xor_sync(0xffffffffu, s, 16);
      n += __shfl_xor_sync(0xffffffffu, n, 16);
      if (mine && h == 0) macc += (T)J.tcc[GD_AT(m, M, kSiteTcc)] * sqrt(s / (T)n);
    } else
    for (int m0 = 32 * my_sub; m0 < M; m0 += 32 * G) {
      const int m = m0 + lane;
      if (m < M) {
        T s = 0;
        int n = 0;
        for (int a = 0; a < L; ++a) {
          const float4 q = J.mcs[GD_AT((size_t)a * M + m, (size_t)L * M, kSiteMcs)];
          if (q.w != 0.0f) {
            const V4<T> la = atom_at(lig, a);
            const T dx = la.x - (T)q.x, dy = la.y - (T)q.y, dz = la.z - (T)q.z;
            s += dx * dx + dy * dy + dz * dz;
            ++n;
          }
        }
        macc += (T)J.tcc[GD_AT(m, M, kSiteTcc)] * sqrt(s / (T)n);
      }
    }
  }
  T elhm = warp_sum(macc);

  if constexpr (SPLIT && PREC != kFP64) {
    if (G > 1) {
      // one replica over G warps: publish this warp's partial sums, and let warp
      // 0 of the group combine them in warp order (compensated for the dense
      // terms with the FP32-Kahan policy) and finish the evaluation
      float *part = sp.gparts + sp.sub * sp.pstride;
      if (lane == 0) {
        part[0] = vdw;
        part[1] = ele;
        part[2] = pmf;
        part[3] = psp;
        part[4] = hdb;
        part[5] = ekde;
        part[6] = elhm;
      }
      group_sync(sp.bar_id, G);
      if (sp.sub != 0) return;
      float cv = 0.f, ce = 0.f, cp = 0.f;
      for (int g = 1; g < G; ++g) {
        const float *o = sp.gparts + g * sp.pstride;
        if constexpr (PREC == kFP32Kahan) {
          kahan_add(vdw, cv, o[0]);
          kahan_add(ele, ce, o[1]);
          kahan_add(pmf, cp, o[2]);
        } else {
          vdw += o[0];
          ele += o[1];
          pmf += o[2];
        }
        psp += o[3];
        hdb += o[4];
        ekde += o[5];
        elhm += o[6];
      }
      vdw += cv;
      ele += ce;
      pmf += cp;
      // the hydrophobic restraint on each atom's combined contact sum (energy_prt_v1.cu:162-169)
      float eh = 0.f;
      for (int a = lane; a < L; a += 32) {
        float S = sp.gparts[kPartTerms + a];
        for (int g = 1; g < G; ++g) S += sp.gparts[g * sp.pstride + kPartTerms + a];
        const int lt = GD_AT(lgrp[GD_AT(a, L, kSiteLgrp)].x, kLigTypes, kSiteTab);
        const float h2 = (S - par->hpl0[lt]) / par->hpl1[lt];
        eh += 0.5f * h2 * h2 - par->hpl2[lt];
      }
      ehpc = warp_sum(eh);
    }
  }

  // ---- distance to the pocket centre, kernel_cuda_l1_montecarlo.cu:439-454
  const float *pc = J.pcenter + 3 * GD_AT(iprt, J.nprt, kSitePrtConf);
  T dst = 0;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T t = ((T)lc[i] + (T)mm[i]) - (T)pc[i];
    dst += t * t;
  }

  T r9[9];
  r9[0] = vdw;
  r9[1] = ele;
  r9[2] = pmf;
  r9[3] = psp;
  r9[4] = hdb * (PREC == kFP64 ? (T)kSqrt2PiInvNegD : (T)kSqrt2PiInvNeg);
  r9[5] = ehpc;
  r9[6] = ekde;
  r9[7] = log(elhm / (T)J.nmcs);
  r9[8] = sqrt(dst);

  // normalisation and weighted total, kernel_cuda_l1_montecarlo.cu:460-476
  if (lane == 0) {
    T tot = 0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      out->raw[i] = (double)r9[i];
      T v = r9[i];
      if (i < 7) v = v / (T)L;
      v = (T)par->a_para[i] * v + (T)par->b_para[i];
      out->e[i] = (double)v;
      tot += (T)par->w[i] * v;
    }
    out->e[9] = (double)tot;
  }
  __syncwarp();
}

// ------------------------------------------------------------ kernels --


// Stage the shared data of work item `wi` into shared memory.  Returns false,
// in every thread of the CTA alike, if the bulk copies did not complete within
// the wait limit; the barrier phase is then left open (see stage_abandon).
template <bool FP64>
__device__ bool stage_item(const KArgs &A, const DevJob &J, const WorkItem &wi, unsigned char *smem,
                           const SmemLayout &sl, uint64_t *bar, uint32_t &phase)
{
  const int P = J.npoint_pad;
  const bool kde_in_smem = J.nkde <= A.Kst;
  const bool pocket_in_smem = A.P > 0;
  if (threadIdx.x == 0) {
    fence_proxy_async_smem();
    const uint32_t pbytes = (uint32_t)(FP64 ? sizeof(DevParams) : kParamScalarBytes);
    uint32_t bytes = pbytes + (pocket_in_smem ? 24u * (uint32_t)P : 0u);
    if (kde_in_smem) bytes += 16u * (uint32_t)J.nkde;
    mbar_expect_tx(bar, bytes + A.stall_bytes);
    bulk_g2s(smem + sl.params, J.par, pbytes, bar);
    if (pocket_in_smem) {
      bulk_g2s(smem + sl.pos, J.pos + (size_t)wi.prt * P, 16u * (uint32_t)P, bar);
      bulk_g2s(smem + sl.aux, J.aux + (size_t)wi.prt * P, 8u * (uint32_t)P, bar);
    }
    if (kde_in_smem && J.nkde > 0) bulk_g2s(smem + sl.kde, J.kde, 16u * (uint32_t)J.nkde, bar);
  }
  int2 *lg = reinterpret_cast<int2 *>(smem + sl.lgrp);
  for (int a = threadIdx.x; a < J.natom; a += blockDim.x) lg[a] = J.lgrp[a];
  // one decision for the whole CTA: a thread that saw the phase complete and
  // one that gave up must not go separate ways
  const bool ok = __syncthreads_and(mbar_wait(bar, phase, wait_limit_ns(A.wait_limit)) ? 1 : 0) != 0;
  phase ^= 1u;
  return ok;
}

// After stage_item gave up: before the CTA returns (and its shared memory goes
// to another CTA), let the copies it issued land.  Bytes the test hook
// announced without a copy are taken off the barrier first, so that the phase
// completes exactly when the real copies have arrived; the wait is bounded
// again.  `phase` is the parity stage_item already advanced.
__device__ void stage_abandon(const KArgs &A, uint64_t *bar, uint32_t phase)
{
  if (threadIdx.x == 0 && A.stall_bytes) mbar_complete_tx(bar, A.stall_bytes);
  __syncthreads();
  (void)__syncthreads_and(mbar_wait(bar, phase ^ 1u, wait_limit_ns(A.wait_limit)) ? 1 : 0);
}

// Per-warp FP64 statistics kept in shared memory during a chunk (lane 0).
struct WarpStats {
  double e_sum, e_sum2, best_e;
  long long n_acc;
  float best_mm[6];
  int best_step;
  int pad_;
};

template <int MODE, int PREC, int KPL, int AB, bool SPLIT = false>
__global__ void __maxnreg__(PREC == kFP64 ? 128 : 80) mc_kernel(KArgs A)
{
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_item;
  // G warps per replica (latency mode, the SPLIT instantiation): warp `sub` of replica slot `gi`
  const int G = SPLIT ? kernel_group<MODE, PREC>(A) : 1;
  const SmemLayout sl = smem_layout(A.P, A.Kst, A.lig_slots, blockDim.x / 32, PREC == kFP64, G);
  const int warp = threadIdx.x >> 5;
  const int lane = lane_id();
  const int gi = warp / G, sub = warp - gi * G;
  // a Complex the device packer refused (gd_devpack.cu) leaves its job unread
  if (*(volatile int *)A.err & kErrPack) return;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  uint32_t phase = 0;
  int prev_job = -1, prev_prt = -1;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(A.queue, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= A.n_items) break;
    const WorkItem wi = A.items[it];
    const DevJob &J = A.jobs[wi.job];
    if (wi.job != prev_job || wi.prt != prev_prt) {
      if (!stage_item<PREC == kFP64>(A, J, wi, smem, sl, &bar, phase)) {
        if (threadIdx.x == 0) atomicOr(A.err, kErrTimeout);
        stage_abandon(A, &bar, phase);
        return;
      }
      if constexpr (PREC != kFP64 && KPL % 2 == 0) {
        __syncthreads();  // type groups are in shared memory
        if (wi.job != prev_job)
          build_pair_tables(J.natom, J.par,
                            reinterpret_cast<const int2 *>(smem + sl.lgrp), reinterpret_cast<float4 *>(smem + sl.apt),
                            reinterpret_cast<float4 *>(smem + sl.aph), reinterpret_cast<int4 *>(smem + sl.ahd));
      }
      prev_job = wi.job;
      prev_prt = wi.prt;
    }
    __syncthreads();
    const float4 *apt = reinterpret_cast<const float4 *>(smem + sl.apt);
    const float4 *aph = reinterpret_cast<const float4 *>(smem + sl.aph);
    const int4 *ahd = reinterpret_cast<const int4 *>(smem + sl.ahd);

    // FP32: only the scalar prefix of DevParams is in shared memory (no table is read through par)
    const DevParams *par = reinterpret_cast<const DevParams *>(smem + sl.params);
    // the protein conformation: staged in shared memory, or read through L1
    const float4 *pos = A.P > 0 ? reinterpret_cast<const float4 *>(smem + sl.pos)
                                : J.pos + (size_t)wi.prt * J.npoint_pad;
    const float2 *aux = A.P > 0 ? reinterpret_cast<const float2 *>(smem + sl.aux)
                                : J.aux + (size_t)wi.prt * J.npoint_pad;
    const float4 *kde = (J.nkde <= A.Kst) ? reinterpret_cast<const float4 *>(smem + sl.kde) : J.kde;
    const int2 *lgrp = reinterpret_cast<const int2 *>(smem + sl.lgrp);
    // each warp rotates the ligand into its own buffer; the replica's state, its
    // proposal and the evaluation's result live in the group's first warp
    unsigned char *wbase = smem + sl.warp0 + (size_t)warp * sl.warp_bytes;
    unsigned char *gbase = smem + sl.warp0 + (size_t)(gi * G) * sl.warp_bytes;
    void *ligbuf = wbase;
    ReplicaMC *srep = reinterpret_cast<ReplicaMC *>(gbase + sl.lig_bytes);
    EnergyScratch *esc = reinterpret_cast<EnergyScratch *>(gbase + sl.lig_bytes + sizeof(ReplicaMC));
    WarpStats *wst = reinterpret_cast<WarpStats *>(gbase + sl.lig_bytes + sizeof(ReplicaMC) + sizeof(EnergyScratch));
    typename std::conditional<SPLIT, Split, NoSplit>::type sp{};
    if constexpr (SPLIT) sp = Split{sub, G, 1 + gi, reinterpret_cast<float *>(gbase + sl.parts), sl.warp_bytes / 4u};
    const bool lead = sub == 0;  // the group's first warp: proposal, Metropolis, state

    if (gi < wi.count) {
      const int r = wi.rep0 + gi;  // job-local index
      if constexpr (MODE == 1) {
        // ---- pose evaluation
        const int ilig = A.conf[2 * r], iprt = A.conf[2 * r + 1];
        if (lane < 6) esc->mm[lane] = A.mm[6 * r + lane];
        __syncwarp();
        energy_warp<PREC, KPL, AB>(J, par, pos, aux, kde, lgrp, apt, aph, ahd, ligbuf, ilig, iprt, esc->mm, esc);
        if (lane < 10) {
          A.out[10 * (size_t)r + lane] = (float)esc->e[lane];
          if (A.out64) A.out64[10 * (size_t)r + lane] = esc->e[lane];
        }
        if (A.raw && lane < 9) A.raw[9 * (size_t)r + lane] = (float)esc->raw[lane];
        __syncwarp();
      } else {
        // ---- Monte Carlo chunk for replica r
        const int gr = J.rid_base + r;
        int *sw = reinterpret_cast<int *>(srep);
        if (lead) sw[lane] = reinterpret_cast<const int *>(J.rep + GD_AT(r, J.nrep, kSiteRep))[lane];
        if (lead && lane == 0) {
          const RepStats &S = J.stats[r];
          wst->e_sum = 0.0;
          wst->e_sum2 = 0.0;
          wst->n_acc = 0;
          wst->best_e = S.best_e;
          wst->best_step = S.best_step;
          for (int i = 0; i < 6; ++i) wst->best_mm[i] = S.best_mm[i];
        }
        __syncwarp();
        if (G > 1) group_sync(1 + gi, G);  // the replica's state is in shared memory
        int acc = J.run_acc[r];
        const int ilig = srep->idx_lig, iprt = srep->idx_prt;
        const double mbeta = (double)J.minus_beta[GD_AT(srep->idx_tmp, J.ntmp, kSiteTmp)];
        Record *rec = (J.rec && (A.flags & kMcRecord)) ? J.rec + r : nullptr;
        int ne = 0;
        if (J.rec && (A.flags & kMcResetRecord)) {
          if (lead && lane == 0) J.rec[r].next_entry = 0;
        } else if (rec) {
          ne = rec->next_entry;
        }
        const bool initial = (A.flags & kMcInitial) != 0;

        const int s0 = (A.d_step ? *A.d_step + A.s_begin : A.s_begin) + J.step0;
        const int nsteps = J.nsteps > 0 ? min(J.nsteps, A.nsteps) : A.nsteps;
        for (int s = s0; s < s0 + nsteps; ++s) {
          if (acc && lead) {
            // record the old state, kernel_cuda_l1_montecarlo.cu:290-297
            if (lane == 0) srep->step = s;
            __syncwarp();
            if (rec && ne < GD_STEPS_PER_DUMP) reinterpret_cast<int *>(&rec->replica[ne])[lane] = sw[lane];
            ++ne;
          }
          // draws of step s: counter {s, replica, 0, 0} -> move x y z, rot x;
          // {s, replica, 0, 1} -> rot y z, accept (lane 0 and lane 1 compute one each)
          float u_acc = 0.0f;
          if (!lead) {
            // the proposal is the group's first warp's
          } else if (!initial) {
            const Philox4 d = philox4x32_10((uint32_t)s, (uint32_t)gr, 0u, (uint32_t)(lane & 1), J.key0, J.key1);
            float u[7];
#pragma unroll
            for (int k = 0; k < 4; ++k) u[k] = u01(__shfl_sync(0xffffffffu, d.v[k], 0));
#pragma unroll
            for (int k = 4; k < 7; ++k) u[k] = u01(__shfl_sync(0xffffffffu, d.v[k - 4], 1));
            u_acc = u[6];
            if (lane < 6) {
              float v = u[0];
#pragma unroll
              for (int i = 1; i < 6; ++i) v = (lane == i) ? u[i] : v;
              esc->mm[lane] = __fmaf_rn(par->move_scale[lane], v, srep->movematrix[lane]);
            }
          } else if (lane < 6) {
            esc->mm[lane] = __fmaf_rn(par->move_scale[lane], 0.0f, srep->movematrix[lane]);
          }
          __syncwarp();
          if (G > 1) group_sync(1 + gi, G);  // the proposal is in shared memory
          energy_warp<PREC, KPL, AB, SPLIT>(J, par, pos, aux, kde, lgrp, apt, aph, ahd, ligbuf, ilig, iprt, esc->mm, esc,
                                            sp);
          if (!lead) continue;  // the group's first warp holds the result
          const float etot = (float)esc->e[9];

          // Metropolis test in FP64, kernel_cuda_l1_montecarlo.cu:485-507
          int accept = 1;
          if (!initial) {
            const double lr = ((double)etot - (double)srep->energy[9]) * mbeta;
            accept = log((double)u_acc) < lr;
          }
          __syncwarp();
          if (accept) {
            if (lane < 10) srep->energy[lane] = (float)esc->e[lane];
            if (lane < 6) srep->movematrix[lane] = esc->mm[lane];
          }
          __syncwarp();
          if (lane == 0) {
            const double ecur = (double)srep->energy[9];
            wst->n_acc += accept;
            wst->e_sum += ecur;
            wst->e_sum2 += ecur * ecur;
            if (wst->best_step < 0 || ecur < wst->best_e) {
              wst->best_e = ecur;
              wst->best_step = s;
              for (int i = 0; i < 6; ++i) wst->best_mm[i] = srep->movematrix[i];
            }
          }
          acc = accept;
        }

        if (lead) {
          if (lane == 0) {
            J.run_acc[r] = acc;
            if (A.flags & kMcStoreAccept) srep->is_accept = acc;
            if (rec) rec->next_entry = ne;
            RepStats &S = J.stats[r];
            S.e_sum += wst->e_sum;
            S.e_sum2 += wst->e_sum2;
            S.n_steps += nsteps;
            S.n_accept += wst->n_acc;
            S.best_e = wst->best_e;
            S.best_step = wst->best_step;
            for (int i = 0; i < 6; ++i) S.best_mm[i] = wst->best_mm[i];
          }
          __syncwarp();
          reinterpret_cast<int *>(J.rep + r)[lane] = sw[lane];
        }
      }
    }
    __syncthreads();
  }
}

// Replica exchange between adjacent temperatures.  Sweep x pairs (t, t+1) for
// t = x mod 2, x mod 2 + 2, ... in every (protein conf p, ligand conf l)
// group; replica index n_tmp*n_lig*p + n_lig*t + l (src/frontend/util.C:380).
// Pair k of the sweep of job J:
__device__ void exchange_one(const DevJob &J, int x, int k)
{
  const int npair = (J.ntmp - (x & 1)) / 2;
  if (npair <= 0) return;
  const int ngroup = J.nprt * J.nlig;
  if (k >= ngroup * npair) return;
  const int g = k / npair, i = k % npair;
  const int p = g / J.nlig, l = g % J.nlig;
  const int t = (x & 1) + 2 * i;
  const int ga = J.ntmp * J.nlig * p + J.nlig * t + l;
  const int gb = ga + J.nlig;
  const int ra = ga - J.rid_base, rb = gb - J.rid_base;
  if (ra < 0 || rb >= J.nrep) return;
  ReplicaMC *A = J.rep + ra, *B = J.rep + rb;
  const Philox4 d = philox4x32_10((uint32_t)x, (uint32_t)g, 1u, (uint32_t)t, J.key0, J.key1);
  const double u = (double)u01(d.v[0]);
  const double ba = -(double)J.minus_beta[t], bb = -(double)J.minus_beta[t + 1];
  const double lr = (ba - bb) * ((double)A->energy[9] - (double)B->energy[9]);
  J.stats[ra].n_exch_try += 1;
  J.stats[rb].n_exch_try += 1;
  if (log(u) < lr) {
#pragma unroll
    for (int q = 0; q < 10; ++q) {
      const float tmp = A->energy[q];
      A->energy[q] = B->energy[q];
      B->energy[q] = tmp;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const float tmp = A->movematrix[q];
      A->movematrix[q] = B->movematrix[q];
      B->movematrix[q] = tmp;
    }
    J.run_acc[ra] = 1;
    J.run_acc[rb] = 1;
    J.stats[ra].n_exch_acc += 1;
    J.stats[rb].n_exch_acc += 1;
  }
}

__global__ void exchange_kernel(const DevJob *jobp, int x)
{
  exchange_one(*jobp, x, blockIdx.x * blockDim.x + threadIdx.x);
}

// One sweep over every job of an ensemble.  xoff[parity][j] is the prefix sum
// of the pair counts (groups x pairs of that parity).  The sweep index is x, or
// with d_step the sweep that ends the chunk [*d_step, *d_step + chunk).
__global__ void exchange_all_kernel(const DevJob *jobs, const int *xoff, int njob, int x, const int *d_step,
                                    int spx, int chunk)
{
  if (d_step) x = (*d_step + chunk) / spx - 1;
  const int *off = xoff + (x & 1) * (njob + 1);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= off[njob]) return;
  int lo = 0, hi = njob;  // off[lo] <= tid < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= tid) lo = mid;
    else hi = mid;
  }
  exchange_one(jobs[lo], x, tid - off[lo]);
}

// One sweep per job with the job's own sweep index (jobs admitted at
// different times are at different steps): blockIdx.y is the job.
__global__ void exchange_jobs_kernel(const DevJob *jobs)
{
  const DevJob &J = jobs[blockIdx.y];
  if (J.xsweep < 0) return;
  exchange_one(J, J.xsweep, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void advance_step_kernel(int *d_step, int n) { *d_step += n; }
__global__ void set_step_kernel(int *d_step, int v) { *d_step = v; }

// Pose evaluation that reads the packed job straight from global memory (no
// shared-memory staging, no work items): warp w of the grid evaluates poses
// w, w + (number of warps), ...  Used by the allocation-free entry point.
template <int PREC, int KPL, int AB>
__global__ void __launch_bounds__(256) eval_global_kernel(const DevJob *jobp, const int *conf, const float *mm,
                                                          int n, float *out, float *raw, int *err)
{
  extern __shared__ __align__(128) unsigned char smem[];
  if (err != nullptr && *(volatile int *)err != 0) return;  // the job was not packed
  const DevJob &J = *jobp;
  const int warp = threadIdx.x >> 5, lane = lane_id();
  const uint32_t lig_bytes = (uint32_t)kMaxAtoms * 32u;
  unsigned char *wb = smem + (size_t)warp * (lig_bytes + sizeof(EnergyScratch));
  EnergyScratch *esc = reinterpret_cast<EnergyScratch *>(wb + lig_bytes);
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  for (int i = blockIdx.x * (blockDim.x >> 5) + warp; i < n; i += nwarps) {
    const int ilig = conf[2 * i], iprt = conf[2 * i + 1];
    if (ilig < 0 || ilig >= J.nlig || iprt < 0 || iprt >= J.nprt) {
      if (lane < 10) out[10 * (size_t)i + lane] = __int_as_float(0x7fc00000);
      if (lane == 0) atomicOr(err, kErrSize);
      continue;
    }
    if (lane < 6) esc->mm[lane] = mm[6 * (size_t)i + lane];
    __syncwarp();
    const size_t P = (size_t)J.npoint_pad;
    // KPL = 1: the per-type-group form, which needs no per-work-item tables
    energy_warp<PREC, KPL, AB>(J, J.par, J.pos + iprt * P, J.aux + iprt * P, J.kde, J.lgrp, nullptr, nullptr, nullptr,
                               wb, ilig, iprt, esc->mm, esc);
    if (lane < 10) out[10 * (size_t)i + lane] = (float)esc->e[lane];
    if (raw && lane < 9) raw[9 * (size_t)i + lane] = (float)esc->raw[lane];
    __syncwarp();
  }
}

cudaError_t launch_eval_global(int precision, const DevJob *d_job, const int *conf, const float *mm, int n,
                               float *out, float *raw, int *err, int grid, cudaStream_t st)
{
  const int threads = 256;
  const size_t smem = (size_t)(threads / 32) * ((size_t)kMaxAtoms * 32 + sizeof(EnergyScratch));
  if (n <= 0) return cudaSuccess;
  if (precision == kFP32)
    eval_global_kernel<kFP32, 1, 8><<<grid, threads, smem, st>>>(d_job, conf, mm, n, out, raw, err);
  else if (precision == kFP32Kahan)
    eval_global_kernel<kFP32Kahan, 1, 8><<<grid, threads, smem, st>>>(d_job, conf, mm, n, out, raw, err);
  else if (precision == kFP64)
    eval_global_kernel<kFP64, 1, 8><<<grid, threads, smem, st>>>(d_job, conf, mm, n, out, raw, err);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}

// ---------------------------------------------------------- launchers --
size_t kernel_smem_bytes(int P, int Kst, int lig_slots, int warps, int precision, int group)
{
  return smem_layout(P, Kst, lig_slots, warps, precision == kFP64, group).total;
}

template <int MODE, int PREC, int KPL, int AB>
static cudaError_t launch_t(const KArgs &a, int warps, int grid, cudaStream_t st)
{
  const int group = kernel_group<MODE, PREC>(a);
  const size_t smem = kernel_smem_bytes(a.P, a.Kst, a.lig_slots, warps, PREC, group);
  auto k = mc_kernel<MODE, PREC, KPL, AB, false>;
  if constexpr (MODE == 0 && PREC != kFP64 && KPL % 2 == 0)
    if (group > 1) k = mc_kernel<MODE, PREC, KPL, AB, true>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, warps * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <int MODE, int PREC>
static cudaError_t launch_p(const KArgs &a, const TileConfig &tc, int grid, cudaStream_t st)
{
  const int w = tc.warps_per_cta;
  if (tc.kpl == 1 && tc.ab == 8) return launch_t<MODE, PREC, 1, 8>(a, w, grid, st);
  if (tc.kpl == 2 && tc.ab == 4) return launch_t<MODE, PREC, 2, 4>(a, w, grid, st);
  if (tc.kpl == 2 && tc.ab == 8) return launch_t<MODE, PREC, 2, 8>(a, w, grid, st);
  if (tc.kpl == 4 && tc.ab == 4) return launch_t<MODE, PREC, 4, 4>(a, w, grid, st);
  if (tc.kpl == 4 && tc.ab == 8) return launch_t<MODE, PREC, 4, 8>(a, w, grid, st);
  return cudaErrorInvalidValue;
}

cudaError_t launch_kernel(int mode, int precision, const TileConfig &tc, const KArgs &a, int grid, cudaStream_t st)
{
  if (mode == 0) {
    if (precision == kFP32) return launch_p<0, kFP32>(a, tc, grid, st);
    if (precision == kFP32Kahan) return launch_p<0, kFP32Kahan>(a, tc, grid, st);
    if (precision == kFP64) return launch_p<0, kFP64>(a, tc, grid, st);
  } else {
    if (precision == kFP32) return launch_p<1, kFP32>(a, tc, grid, st);
    if (precision == kFP32Kahan) return launch_p<1, kFP32Kahan>(a, tc, grid, st);
    if (precision == kFP64) return launch_p<1, kFP64>(a, tc, grid, st);
  }
  return cudaErrorInvalidValue;
}

int kernel_occupancy(int mode, int precision, const TileConfig &tc, size_t smem)
{
  const void *f = nullptr;
  const bool split = mode == 0 && precision != kFP64 && tc.group > 1;
#define GD_PICK(M, PR, K, A)                                                                  \
  if (mode == M && precision == PR && tc.kpl == K && tc.ab == A)                              \
    f = split ? (const void *)mc_kernel<M, PR, K, A, (M == 0 && PR != kFP64 && K % 2 == 0)> \
              : (const void *)mc_kernel<M, PR, K, A, false>;
#define GD_PICK_ALL(M, PR) \
  GD_PICK(M, PR, 1, 8) GD_PICK(M, PR, 2, 4) GD_PICK(M, PR, 2, 8) GD_PICK(M, PR, 4, 4) GD_PICK(M, PR, 4, 8)
  GD_PICK_ALL(0, kFP32) GD_PICK_ALL(0, kFP32Kahan) GD_PICK_ALL(0, kFP64)
  GD_PICK_ALL(1, kFP32) GD_PICK_ALL(1, kFP32Kahan) GD_PICK_ALL(1, kFP64)
#undef GD_PICK_ALL
#undef GD_PICK
  if (!f) return 0;
  if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, tc.warps_per_cta * 32, smem) != cudaSuccess) return 0;
  return nb;
}

cudaError_t launch_exchange_all(const DevJob *d_jobs, const int *d_xoff, int njob, int total, int x,
                                const int *d_step, int spx, int chunk, cudaStream_t st)
{
  if (total <= 0) return cudaSuccess;
  exchange_all_kernel<<<(total + 255) / 256, 256, 0, st>>>(d_jobs, d_xoff, njob, x, d_step, spx, chunk);
  return cudaGetLastError();
}

cudaError_t launch_exchange_jobs(const DevJob *d_jobs, int njob, int max_pairs, cudaStream_t st)
{
  if (njob <= 0 || max_pairs <= 0) return cudaSuccess;
  exchange_jobs_kernel<<<dim3((max_pairs + 127) / 128, njob), 128, 0, st>>>(d_jobs);
  return cudaGetLastError();
}

cudaError_t launch_set_step(int *d_step, int v, cudaStream_t st)
{
  set_step_kernel<<<1, 1, 0, st>>>(d_step, v);
  return cudaGetLastError();
}

cudaError_t launch_advance_step(int *d_step, int n, cudaStream_t st)
{
  advance_step_kernel<<<1, 1, 0, st>>>(d_step, n);
  return cudaGetLastError();
}

cudaError_t launch_exchange(const DevJob *d_job, int ngroup, int ntmp, int x, cudaStream_t st)
{
  const int npair = (ntmp - (x & 1)) / 2;
  if (npair <= 0 || ngroup <= 0) return cudaSuccess;
  const int n = ngroup * npair;
  exchange_kernel<<<(n + 255) / 256, 256, 0, st>>>(d_job, x);
  return cudaGetLastError();
}

}  // namespace gd

// Bounds-check record of the debug build: out4 = {1 if an index was out of
// range, its site (gd::CheckSite), the index, the array length}; reset != 0
// clears it.  The product build returns GD_E_STATE.
extern "C" int gd_check_report(int *out4, int reset)
{
  if (!out4) return gd::fail(GD_E_INVALID, "null argument");
#ifdef GD_CHECK
  GD_CUDA(cudaDeviceSynchronize());
  GD_CUDA(cudaMemcpyFromSymbol(out4, gd::g_check, 4 * sizeof(int)));
  if (reset) {
    const int z[4] = {0, 0, 0, 0};
    GD_CUDA(cudaMemcpyToSymbol(gd::g_check, z, sizeof z));
  }
  return GD_OK;
#else
  (void)reset;
  for (int i = 0; i < 4; ++i) out4[i] = 0;
  return gd::fail(GD_E_STATE, "not a bounds-checking build (libgdock_check.so is built with -DGD_CHECK)");
#endif
}
