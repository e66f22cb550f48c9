// gd_pack.cu -- from the reference Complex (or a cap-free job description)
// to the packed device layout of gd_internal.h.
//
// The packing keeps the semantics of the reference's own SoA re-layout
// (src/frontend/util_optimize_soa.C): KDE points sorted by type (:336-372),
// protein points re-ordered (the reference sorts by class, :236-267; here by
// point type), per-point hpp and ele already resolved (:198-217), and the
// force-field tables of OptimizeEnepara (:489-540).  Two table entries that
// the reference guards with branches are folded into zeros: hdb0/hdb1 of pairs
// with hdb0 <= 0.1 (energy_prt_v1.cu:134, hdb1 = 1/0 there) and the psp value
// of points that are not class 2 (energy_prt_v1.cu:109).
#include <atomic>
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "gd_pack.h"

namespace gd {

namespace {
thread_local std::string t_err;

size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

// A list of (host source, device offset, bytes) copied in one transfer.
struct Arena {
  size_t off = 0;
  std::vector<unsigned char> host;
  size_t take(size_t bytes)
  {
    const size_t o = off;
    off = al256(off + bytes);
    if (host.size() < off) host.resize(off, 0);
    return o;
  }
  template <typename T>
  size_t put(const std::vector<T> &v)
  {
    const size_t o = take(v.size() * sizeof(T));
    if (!v.empty()) std::memcpy(host.data() + o, v.data(), v.size() * sizeof(T));
    return o;
  }
};

inline float as_float(int i)
{
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
inline int as_int(float f)
{
  int i;
  std::memcpy(&i, &f, 4);
  return i;
}
}  // namespace

namespace {
double now_ms()
{
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

Tracer::Tracer(const char *sc) : on(std::getenv("GDOCK_TRACE") != nullptr), scope(sc), t_last(now_ms()) {}

void Tracer::mark(const char *phase)
{
  if (!on) return;
  const double t = now_ms();
  std::fprintf(stderr, "[gdock] %s %-24s %9.3f ms\n", scope, phase, t - t_last);
  t_last = t;
}

int fail(int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
  return code;
}

}  // namespace gd

extern "C" const char *gd_last_error(void) { return gd::t_err.c_str(); }

namespace gd {
namespace {
std::atomic<int> g_fail_alloc{0};
}
void set_injected_alloc_failures(int n) { g_fail_alloc.store(n); }
int injected_alloc_failures() { return g_fail_alloc.load(); }
bool take_injected_alloc_failure()
{
  int n = g_fail_alloc.load();
  while (n > 0)
    if (g_fail_alloc.compare_exchange_weak(n, n - 1)) return true;
  return false;
}
}  // namespace gd

namespace gd {

void default_replicas(int nlig, int nprt, int ntmp, std::vector<ReplicaMC> &out)
{
  out.assign((size_t)nlig * nprt * ntmp, ReplicaMC{});
  for (int p = 0; p < nprt; ++p)
    for (int t = 0; t < ntmp; ++t)
      for (int l = 0; l < nlig; ++l) {
        const int r = ntmp * nlig * p + nlig * t + l;
        ReplicaMC &R = out[r];
        std::memset(&R, 0, sizeof(R));
        R.idx_rep = r;
        R.idx_prt = p;
        R.idx_tmp = t;
        R.idx_lig = l;
      }
}

int pocket_from_complex(const Complex *c, PocketData &pk)
{
  const int nprt = c->size.n_prt;
  if (nprt < 1 || nprt > GD_MAX_CONF_PRT)
    return fail(GD_E_INVALID, "n_prt = %d outside [1, %d]", nprt, GD_MAX_CONF_PRT);
  int P = 0;
  for (int i = 0; i < nprt; ++i) {
    const int n = c->prt[i].prt_npoint;
    if (n < 1 || n > GD_MAXPRO)
      return fail(GD_E_INVALID, "protein conformation %d: prt_npoint = %d outside [1, %d]", i, n, GD_MAXPRO);
    P = std::max(P, n);
  }
  pk = PocketData{};
  pk.nconf = nprt;
  pk.P = P;
  pk.hdb_types = hdb_point_types(c->enepara);
  pk.npts.resize(nprt);
  pk.xyz.assign((size_t)nprt * P * 3, 0.f);
  pk.type.assign((size_t)nprt * P, 0);
  pk.cls.assign((size_t)nprt * P, 0);
  pk.cdc.assign((size_t)nprt * P, 0);
  pk.seq3r.assign((size_t)nprt * P, 0);
  pk.hpp.assign((size_t)nprt * P, 0.f);
  pk.ele.assign((size_t)nprt * P, 0.f);
  pk.center.resize((size_t)nprt * 3);
  for (int i = 0; i < nprt; ++i) {
    const Protein &pr = c->prt[i];
    pk.npts[i] = pr.prt_npoint;
    for (int k = 0; k < pr.prt_npoint; ++k) {
      const size_t o = (size_t)i * P + k;
      pk.xyz[3 * o + 0] = pr.x[k];
      pk.xyz[3 * o + 1] = pr.y[k];
      pk.xyz[3 * o + 2] = pr.z[k];
      pk.type[o] = pr.t[k];
      pk.cls[o] = pr.c[k];
      pk.cdc[o] = pr.cdc[k];
      pk.seq3r[o] = pr.seq3r[k];
      pk.hpp[o] = pr.hpp[k];
      pk.ele[o] = pr.ele[k];
    }
    for (int d = 0; d < 3; ++d) pk.center[3 * i + d] = pr.pocket_center[d];
  }
  return GD_OK;
}

int job_from_complex(const Complex *c, int rep_begin, int rep_end, uint64_t seed, JobData &jd)
{
  const ComplexSize &sz = c->size;
  if (sz.n_lig < 1 || sz.n_lig > GD_MAX_CONF_LIG)
    return fail(GD_E_INVALID, "n_lig = %d outside [1, %d]", sz.n_lig, GD_MAX_CONF_LIG);
  if (sz.n_tmp < 1 || sz.n_tmp > GD_MAX_TMP)
    return fail(GD_E_INVALID, "n_tmp = %d outside [1, %d]", sz.n_tmp, GD_MAX_TMP);
  if (sz.n_prt < 1 || sz.n_prt > GD_MAX_CONF_PRT)
    return fail(GD_E_INVALID, "n_prt = %d outside [1, %d]", sz.n_prt, GD_MAX_CONF_PRT);
  if (sz.n_rep < 1 || sz.n_rep > GD_MAX_REP)
    return fail(GD_E_INVALID, "n_rep = %d outside [1, %d]", sz.n_rep, GD_MAX_REP);
  if (rep_begin < 0 || rep_end >= sz.n_rep || rep_begin > rep_end)
    return fail(GD_E_INVALID, "replica range [%d, %d] outside [0, %d)", rep_begin, rep_end, sz.n_rep);
  const int L = c->lig[0].lig_natom;
  if (L < 1 || L > GD_MAXLIG) return fail(GD_E_INVALID, "lig_natom = %d outside [1, %d]", L, GD_MAXLIG);
  jd = JobData{};
  jd.L = L;
  jd.nlig = sz.n_lig;
  jd.nprt = sz.n_prt;
  jd.lxyz.resize((size_t)sz.n_lig * L * 3);
  jd.lcenter.resize((size_t)sz.n_lig * 3);
  for (int i = 0; i < sz.n_lig; ++i) {
    const Ligand &lg = c->lig[i];
    if (lg.lig_natom != L)
      return fail(GD_E_INVALID, "ligand conformation %d has %d atoms, conformation 0 has %d", i, lg.lig_natom, L);
    for (int a = 0; a < L; ++a) {
      jd.lxyz[((size_t)i * L + a) * 3 + 0] = lg.x2[a];
      jd.lxyz[((size_t)i * L + a) * 3 + 1] = lg.y2[a];
      jd.lxyz[((size_t)i * L + a) * 3 + 2] = lg.z2[a];
    }
    for (int d = 0; d < 3; ++d) jd.lcenter[3 * i + d] = lg.center[d];
  }
  jd.ltype.assign(c->lig[0].t2, c->lig[0].t2 + L);
  jd.lcharge.assign(c->lig[0].c2, c->lig[0].c2 + L);

  jd.K = sz.kde_npoint;
  if (jd.K < 0 || jd.K > GD_MAXKDE) return fail(GD_E_INVALID, "kde_npoint = %d outside [0, %d]", jd.K, GD_MAXKDE);
  jd.kxyz.resize((size_t)jd.K * 3);
  jd.ktype.resize(jd.K);
  for (int k = 0; k < jd.K; ++k) {
    jd.kxyz[3 * k + 0] = c->kde.x[k];
    jd.kxyz[3 * k + 1] = c->kde.y[k];
    jd.kxyz[3 * k + 2] = c->kde.z[k];
    jd.ktype[k] = c->kde.t[k];
  }

  jd.M = sz.mcs_nrow;
  if (jd.M < 1 || jd.M > GD_MAX_MCS_ROW)
    return fail(GD_E_INVALID, "mcs_nrow = %d outside [1, %d]", jd.M, GD_MAX_MCS_ROW);
  jd.mxyz.resize((size_t)jd.M * L * 3);
  jd.tcc.resize(jd.M);
  for (int m = 0; m < jd.M; ++m) {
    for (int a = 0; a < L; ++a) {
      jd.mxyz[((size_t)m * L + a) * 3 + 0] = c->mcs[m].x[a];
      jd.mxyz[((size_t)m * L + a) * 3 + 1] = c->mcs[m].y[a];
      jd.mxyz[((size_t)m * L + a) * 3 + 2] = c->mcs[m].z[a];
    }
    jd.tcc[m] = c->mcs[m].tcc;
  }

  jd.psp_ncol = GD_MAXPRO;
  jd.psp.resize((size_t)kLigTypes * GD_MAXPRO);
  for (int t = 0; t < kLigTypes; ++t) std::memcpy(&jd.psp[(size_t)t * GD_MAXPRO], c->psp.psp[t], sizeof(float) * GD_MAXPRO);

  jd.ntmp = sz.n_tmp;
  jd.minus_beta.resize(sz.n_tmp);
  for (int t = 0; t < sz.n_tmp; ++t) jd.minus_beta[t] = c->temp[t].minus_beta;
  for (int i = 0; i < 6; ++i) jd.move_scale[i] = c->mcpara.move_scale[i];
  jd.seed = seed;

  jd.rid_base = rep_begin;
  jd.nrep_total = sz.n_rep;
  jd.reps.assign(c->replica + rep_begin, c->replica + rep_end + 1);
  for (size_t i = 0; i < jd.reps.size(); ++i) {
    const ReplicaMC &R = jd.reps[i];
    if (R.idx_lig < 0 || R.idx_lig >= sz.n_lig || R.idx_prt < 0 || R.idx_prt >= sz.n_prt || R.idx_tmp < 0 ||
        R.idx_tmp >= sz.n_tmp)
      return fail(GD_E_INVALID, "replica %d: indices (lig %d, prt %d, tmp %d) out of range", rep_begin + (int)i,
                  R.idx_lig, R.idx_prt, R.idx_tmp);
  }
  return GD_OK;
}

int pocket_from_desc(const gd_pocket_desc_t &d, PocketData &pk)
{
  if (d.npoint < 1 || d.nconf < 1) return fail(GD_E_INVALID, "pocket: npoint = %d, nconf = %d", d.npoint, d.nconf);
  if (!d.xyz || !d.type || !d.cls || !d.cdc || !d.seq3r || !d.hpp || !d.ele || !d.center)
    return fail(GD_E_INVALID, "pocket: null array");
  const int P = d.npoint, n = d.nconf;
  pk = PocketData{};
  pk.nconf = n;
  pk.P = P;
  pk.npts.assign(n, P);
  pk.xyz.assign(d.xyz, d.xyz + (size_t)n * P * 3);
  pk.center.assign(d.center, d.center + (size_t)n * 3);
  pk.type.resize((size_t)n * P);
  pk.cls.resize((size_t)n * P);
  pk.cdc.resize((size_t)n * P);
  pk.seq3r.resize((size_t)n * P);
  pk.hpp.resize((size_t)n * P);
  pk.ele.resize((size_t)n * P);
  for (int i = 0; i < n; ++i) {
    std::copy(d.type, d.type + P, pk.type.begin() + (size_t)i * P);
    std::copy(d.cls, d.cls + P, pk.cls.begin() + (size_t)i * P);
    std::copy(d.cdc, d.cdc + P, pk.cdc.begin() + (size_t)i * P);
    std::copy(d.seq3r, d.seq3r + P, pk.seq3r.begin() + (size_t)i * P);
    std::copy(d.hpp, d.hpp + P, pk.hpp.begin() + (size_t)i * P);
    std::copy(d.ele, d.ele + P, pk.ele.begin() + (size_t)i * P);
  }
  return GD_OK;
}

int job_from_desc(const gd_job_desc_t &d, int nprt, JobData &jd)
{
  if (d.natom < 1 || d.natom > kMaxAtoms)
    return fail(GD_E_CAPACITY, "job: natom = %d outside [1, %d]", d.natom, kMaxAtoms);
  if (d.nlig < 1 || d.ntmp < 1 || d.nmcs < 1 || d.nkde < 0 || d.psp_ncol < 1)
    return fail(GD_E_INVALID, "job: nlig = %d, ntmp = %d, nmcs = %d, nkde = %d, psp_ncol = %d", d.nlig, d.ntmp, d.nmcs,
                d.nkde, d.psp_ncol);
  if (!d.lig_xyz || !d.lig_type || !d.lig_charge || !d.lig_center || !d.mcs_xyz || !d.mcs_tcc || !d.psp ||
      !d.temperature || (d.nkde > 0 && (!d.kde_xyz || !d.kde_type)))
    return fail(GD_E_INVALID, "job: null array");
  const int L = d.natom;
  jd = JobData{};
  jd.L = L;
  jd.nlig = d.nlig;
  jd.nprt = nprt;
  jd.lxyz.assign(d.lig_xyz, d.lig_xyz + (size_t)d.nlig * L * 3);
  jd.ltype.assign(d.lig_type, d.lig_type + L);
  jd.lcharge.assign(d.lig_charge, d.lig_charge + L);
  jd.lcenter.assign(d.lig_center, d.lig_center + (size_t)d.nlig * 3);
  jd.K = d.nkde;
  jd.kxyz.assign(d.kde_xyz, d.kde_xyz + (size_t)d.nkde * 3);
  jd.ktype.assign(d.kde_type, d.kde_type + d.nkde);
  jd.M = d.nmcs;
  jd.mxyz.assign(d.mcs_xyz, d.mcs_xyz + (size_t)d.nmcs * L * 3);
  jd.tcc.assign(d.mcs_tcc, d.mcs_tcc + d.nmcs);
  jd.psp_ncol = d.psp_ncol;
  jd.psp.assign(d.psp, d.psp + (size_t)kLigTypes * d.psp_ncol);
  jd.ntmp = d.ntmp;
  jd.minus_beta.resize(d.ntmp);
  for (int t = 0; t < d.ntmp; ++t) {
    if (!(d.temperature[t] > 0.f)) return fail(GD_E_INVALID, "job: temperature[%d] = %g", t, d.temperature[t]);
    // SetTemperature, src/frontend/util.C:346-351: beta = 1/(k_B T), k_B = 1
    const float beta = 1.0f / (1.0f * d.temperature[t]);
    jd.minus_beta[t] = 0.0f - beta;
  }
  for (int i = 0; i < 6; ++i) jd.move_scale[i] = d.move_scale[i];
  jd.seed = d.seed;
  default_replicas(d.nlig, nprt, d.ntmp, jd.reps);
  jd.rid_base = 0;
  jd.nrep_total = (int)jd.reps.size();
  return GD_OK;
}

uint32_t hdb_point_types(const EnePara &ep)
{
  uint32_t m = 0;
  for (int lt = 0; lt < kLigTypes; ++lt)
    for (int pt = 0; pt < kPadType; ++pt)
      if (ep.hdb0[lt][pt] > 0.1f) m |= 1u << pt;
  return m;
}

int build_params(const EnePara &ep, const float move_scale[6], DevParams &p)
{
  std::memset(&p, 0, sizeof(p));
  const double c = kHdbC;
  for (int lt = 0; lt < kLigTypes; ++lt) {
    for (int pt = kPadType; pt < kTabCols; ++pt) p.tab4[lt][pt] = tab4_padding();
    for (int pt = 0; pt < GD_MAXTP1 && pt < kPadType; ++pt) {
      if (!(ep.p1a[lt][pt] > 0.f))
        return fail(GD_E_INVALID, "enepara: p1a[%d][%d] = %g (the pair kernel needs p1a > 0)", lt, pt,
                    (double)ep.p1a[lt][pt]);
      p.tab4[lt][pt] = tab4_entry(ep.p1a[lt][pt], ep.p2a[lt][pt], ep.pmf0[lt][pt], ep.pmf1[lt][pt]);
      // energy_prt_v1.cu:133-138 evaluates the hydrogen-bond term only where hdb0 > 0.1
      const float h0 = ep.hdb0[lt][pt], h1 = ep.hdb1[lt][pt];
      if (h0 > 0.1f) {
        p.tab2[lt][pt] = make_float2((float)((double)h1 * c), (float)(-(double)h0 * (double)h1 * c));
        p.hdbmask[lt] |= 1u << pt;
      } else {
        p.tab2[lt][pt] = make_float2(0.f, 0.f);
      }
    }
    p.hpl0[lt] = ep.hpl0[lt];
    p.hpl1[lt] = ep.hpl1[lt];
    p.hpl2[lt] = ep.hpl2[lt];
  }
  for (int i = 0; i < GD_MAXWEI; ++i) {
    p.a_para[i] = ep.a_para[i];
    p.b_para[i] = ep.b_para[i];
    p.w[i] = ep.w[i];
  }
  p.lj0 = ep.lj0;
  p.lj1 = ep.lj1;
  p.el0 = ep.el0;
  p.el1 = ep.el1;
  p.inv_el1 = 1.0f / ep.el1;
  p.a1 = ep.a1;
  p.b1 = ep.b1;
  p.kde2 = ep.kde2;
  p.kde3_inv = 1.0f / ep.kde3;  // kernel_cuda_l1_montecarlo.cu:194
  p.kde3 = ep.kde3;
  p.lj01 = (float)((double)ep.lj0 * ep.lj1);
  p.ele_a = (float)((double)ep.a1 * ep.el1 * ep.el1);
  p.ele_b = (float)((double)ep.b1 * ep.el1 * ep.el1 * ep.el1);
  p.ele_d2max = (float)(1.0 / ((double)ep.el1 * ep.el1));
  p.hdb_cinv = (float)(1.0 / c);
  for (int i = 0; i < 6; ++i) p.move_scale[i] = move_scale[i];
  return GD_OK;
}

int pack_pocket(const PocketData &pk, DevPocket &out, const DevPocket *reuse, cudaStream_t st)
{
  out = DevPocket{};
  const int n = pk.nconf;
  const int Ppad = ((std::max(pk.P, 1) + kPointAlign - 1) / kPointAlign) * kPointAlign;
  out.nconf = n;
  out.Ppad = Ppad;
  out.hdb_types = pk.hdb_types;
  std::vector<float4> pos((size_t)n * Ppad);
  std::vector<float2> aux((size_t)n * Ppad);
  std::vector<int> ncdc(n, 0);
  out.scls.assign((size_t)n * Ppad, -1);
  out.sseq.assign((size_t)n * Ppad, 0);
  out.stype.assign((size_t)n * Ppad, kPadType);
  for (int i = 0; i < n; ++i) {
    const int np = pk.npts[i];
    std::vector<int> idx(np);
    std::iota(idx.begin(), idx.end(), 0);
    for (int k = 0; k < np; ++k) {
      const int t = pk.type[(size_t)i * pk.P + k];
      if (t < 0 || t >= kPadType) return fail(GD_E_INVALID, "protein conformation %d point %d: type %d outside [0, %d)", i, k, t, kPadType);
    }
    // hydrophobic-contact points first (their rows are the only ones the
    // hydrophobic term visits); in each part the point types with a
    // hydrogen-bond parameter first (the pair loop evaluates that term only for
    // rows holding such a type), each group sorted by point type
    auto key = [&](int k) {
      const size_t o = (size_t)i * pk.P + k;
      const int t = pk.type[o];
      return (pk.cdc[o] == 1 ? 0 : 64) + (((pk.hdb_types >> t) & 1u) ? 0 : 32) + t;
    };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key(a) < key(b); });
    int nc = 0;
    for (int k = 0; k < np; ++k) nc += pk.cdc[(size_t)i * pk.P + k] == 1;
    ncdc[i] = nc;
    for (int j = 0; j < Ppad; ++j) {
      const size_t o = (size_t)i * Ppad + j;
      if (j < np) {
        const size_t s = (size_t)i * pk.P + idx[j];
        pos[o] = make_float4(pk.xyz[3 * s], pk.xyz[3 * s + 1], pk.xyz[3 * s + 2], pk.ele[s]);
        // hydrophobic contact applies to cdc == 1 points only (energy_prt_v1.cu:42)
        aux[o] = make_float2(pk.cdc[s] == 1 ? pk.hpp[s] : 0.f, as_float(pk.type[s]));
        out.scls[o] = pk.cls[s];
        out.sseq[o] = pk.seq3r[s];
        out.stype[o] = pk.type[s];
      } else {
        // inert padding: far away, zero parameters, point type kPadType (all-zero table column)
        pos[o] = make_float4(1.0e4f + (float)j, 1.0e4f, 1.0e4f, 0.f);
        aux[o] = make_float2(0.f, as_float(kPadType));
      }
    }
  }
  out.spos = pos;
  Arena ar;
  const size_t o_pos = ar.put(pos), o_aux = ar.put(aux), o_c = ar.put(pk.center), o_n = ar.put(ncdc);
  if (reuse && reuse->arena && reuse->bytes == ar.off) {
    out.arena = reuse->arena;
    GD_CUDA(cudaMemcpyAsync(out.arena, ar.host.data(), ar.off, cudaMemcpyHostToDevice, st));
  } else {
    GD_CUDA(cudaMalloc(&out.arena, ar.off));
    GD_CUDA(cudaMemcpy(out.arena, ar.host.data(), ar.off, cudaMemcpyHostToDevice));
  }
  out.bytes = ar.off;
  unsigned char *b = (unsigned char *)out.arena;
  out.pos = (float4 *)(b + o_pos);
  out.aux = (float2 *)(b + o_aux);
  out.center = (float *)(b + o_c);
  out.ncdc = (int *)(b + o_n);
  return GD_OK;
}

namespace {
int pack_job_impl(const JobData &jd, const DevPocket &pk, const EnePara &ep, bool want_records, Record *rec,
                  cudaStream_t st, bool async, DevJobBuf &out, const DevJobBuf *reuse = nullptr)
{
  out = DevJobBuf{};
  const int L = jd.L;
  if (L < 1 || L > kMaxAtoms) return fail(GD_E_CAPACITY, "ligand of %d atoms (limit %d)", L, kMaxAtoms);
  if (jd.nprt != pk.nconf)
    return fail(GD_E_INVALID, "job expects %d protein conformations, pocket has %d", jd.nprt, pk.nconf);
  for (int a = 0; a < L; ++a)
    if (jd.ltype[a] < 0 || jd.ltype[a] >= kLigTypes)
      return fail(GD_E_INVALID, "ligand atom %d: type %d outside [0, %d)", a, jd.ltype[a], kLigTypes);

  // atoms grouped by type (stable), as the reference's sorted copy (util_optimize_soa.C:112-126),
  // with the types that have a hydrogen-bond parameter first (an atom pair of the pair loop then
  // mixes such a type with one without at most once)
  uint32_t lhdb = 0;
  for (int lt = 0; lt < kLigTypes; ++lt)
    for (int pt = 0; pt < kPadType; ++pt)
      if (ep.hdb0[lt][pt] > 0.1f) lhdb |= 1u << lt;
  auto lkey = [&](int t) { return (((lhdb >> t) & 1u) ? 0 : 32) + t; };
  std::vector<int> perm(L);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return lkey(jd.ltype[a]) < lkey(jd.ltype[b]); });
  const int lstride = (L + 3) & ~3;
  std::vector<float4> lig((size_t)jd.nlig * lstride, make_float4(0, 0, 0, 0));
  for (int i = 0; i < jd.nlig; ++i)
    for (int a = 0; a < L; ++a) {
      const int s = perm[a];
      const float *x = &jd.lxyz[((size_t)i * L + s) * 3];
      lig[(size_t)i * lstride + a] = make_float4(x[0], x[1], x[2], jd.lcharge[s]);
    }
  std::vector<int> ltype(L), lgend(L);
  for (int a = 0; a < L; ++a) ltype[a] = jd.ltype[perm[a]];
  for (int a = L - 1; a >= 0; --a) lgend[a] = (a + 1 < L && ltype[a + 1] == ltype[a]) ? lgend[a + 1] : a + 1;
  std::vector<int2> lgrp(L);
  for (int a = 0; a < L; ++a) lgrp[a] = make_int2(ltype[a], lgend[a]);

  // KDE: only points with a ligand type can match (getLigCode returns 50 for others)
  std::vector<int> kidx;
  for (int k = 0; k < jd.K; ++k)
    if (jd.ktype[k] >= 0 && jd.ktype[k] < kLigTypes) kidx.push_back(k);
  std::stable_sort(kidx.begin(), kidx.end(), [&](int a, int b) { return jd.ktype[a] < jd.ktype[b]; });
  std::vector<float4> kde(std::max<size_t>(kidx.size(), 1), make_float4(0, 0, 0, 0));
  int kbeg[kLigTypes], kcnt[kLigTypes];
  for (int t = 0; t < kLigTypes; ++t) kbeg[t] = kcnt[t] = 0;
  for (size_t j = 0; j < kidx.size(); ++j) {
    const int k = kidx[j], t = jd.ktype[k];
    kde[j] = make_float4(jd.kxyz[3 * k], jd.kxyz[3 * k + 1], jd.kxyz[3 * k + 2], as_float(t));
    if (kcnt[t] == 0) kbeg[t] = (int)j;
    ++kcnt[t];
  }
  // KDE slots: for each ligand type group (grouped order), each KDE point of its type
  std::vector<int4> kslot;
  for (int a = 0; a < L;) {
    const int t = ltype[a], e = lgend[a];
    if (kcnt[t] > 0) {
      const float inv = 1.0f / (float)kcnt[t];
      for (int k = kbeg[t]; k < kbeg[t] + kcnt[t]; ++k) {
        kslot.push_back(make_int4(as_int(kde[k].x), as_int(kde[k].y), as_int(kde[k].z), as_int(inv)));
        kslot.push_back(make_int4(a | (e << 16), 0, 0, 0));
      }
    }
    a = e;
  }
  const int nkslot = (int)(kslot.size() / 2);
  // room for any ligand of the same shapes (a refill on the GPU): one slot per KDE point
  kslot.resize(2 * (size_t)std::max<size_t>(kidx.size(), 1), make_int4(0, 0, 0, 0));

  // MCS templates, atom-major in grouped order; validity as energy_mcs_v1.cu:295
  std::vector<float4> mcs((size_t)L * jd.M);
  for (int m = 0; m < jd.M; ++m) {
    int nvalid = 0;
    for (int a = 0; a < L; ++a) {
      const float *x = &jd.mxyz[((size_t)m * L + perm[a]) * 3];
      const bool valid = x[0] != GD_MCS_INVALID_COORD;
      nvalid += valid;
      mcs[(size_t)a * jd.M + m] = make_float4(x[0], x[1], x[2], valid ? 1.f : 0.f);
    }
    if (nvalid == 0)
      return fail(GD_E_INVALID, "MCS row %d has no coordinate for any of the %d ligand atoms", m, L);
  }

  // pocket-specific potential gathered per sorted point: psp[t][seq3r] for class 2 points
  const int P = pk.Ppad;
  std::vector<float> psp((size_t)pk.nconf * kLigTypes * P, 0.f);
  std::vector<uint32_t> pspmask((size_t)pk.nconf * P, 0u);
  for (int i = 0; i < pk.nconf; ++i)
    for (int j = 0; j < P; ++j) {
      const size_t o = (size_t)i * P + j;
      if (pk.scls[o] != 2) continue;
      const int col = pk.sseq[o];
      if (col < 0 || col >= jd.psp_ncol)
        return fail(GD_E_INVALID, "protein point with residue serial %d outside the psp table [0, %d)", col,
                    jd.psp_ncol);
      for (int t = 0; t < kLigTypes; ++t) {
        const float v = jd.psp[(size_t)t * jd.psp_ncol + col];
        psp[((size_t)i * kLigTypes + t) * P + j] = v;
        if (v != 0.f) pspmask[o] |= 1u << t;
      }
    }

  DevParams par;
  GD_TRY(build_params(ep, jd.move_scale, par));

  // the same as non-zero cells per conformation for the ligand's types, by type then point
  // (the batched kernel's pocket-specific pass), two int4 per cell: (x, y, z of the point,
  // value) and (beg | end << 16, -pmf0 of (type, point type), type, point), at a stride of
  // the largest count or, with jd.cell_room, of every point times every type the ligand can
  // have (a refill on the GPU of the same shapes always fits)
  int tbeg[kLigTypes], tend[kLigTypes];
  for (int t = 0; t < kLigTypes; ++t) tbeg[t] = tend[t] = 0;
  uint32_t ligmask = 0u;
  for (int a = L - 1; a >= 0; --a) {
    tbeg[ltype[a]] = a;
    if (tend[ltype[a]] == 0) tend[ltype[a]] = a + 1;
    ligmask |= 1u << ltype[a];
  }
  // per conformation: per-type counts, then each cell at its type's running offset
  std::vector<int> pcell_cnt(pk.nconf, 0);
  std::vector<int> tcell((size_t)pk.nconf * kLigTypes, 0);
  for (int i = 0; i < pk.nconf; ++i)
    for (int j = 0; j < P; ++j)
      for (uint32_t m = pspmask[(size_t)i * P + j] & ligmask; m; m &= m - 1u) ++tcell[(size_t)i * kLigTypes + __builtin_ctz(m)];
  int cstride = jd.cell_room ? P * std::min(L, kLigTypes) : 1;
  for (int i = 0; i < pk.nconf; ++i) {
    for (int t = 0; t < kLigTypes; ++t) pcell_cnt[i] += tcell[(size_t)i * kLigTypes + t];
    cstride = std::max(cstride, pcell_cnt[i]);
  }
  std::vector<int4> pcell((size_t)pk.nconf * cstride * 2, make_int4(0, 0, 0, 0));
  for (int i = 0; i < pk.nconf; ++i) {
    int at[kLigTypes];
    for (int t = 0, o = 0; t < kLigTypes; ++t) {
      at[t] = o;
      o += tcell[(size_t)i * kLigTypes + t];
    }
    int4 *cell = pcell.data() + (size_t)i * cstride * 2;
    for (int j = 0; j < P; ++j)
      for (uint32_t m = pspmask[(size_t)i * P + j] & ligmask; m; m &= m - 1u) {
        const int t = __builtin_ctz(m);
        const size_t o = (size_t)i * P + j;
        const float4 q = pk.spos[o];
        const float v = psp[((size_t)i * kLigTypes + t) * P + j];
        const int k = at[t]++;
        cell[2 * k] = make_int4(as_int(q.x), as_int(q.y), as_int(q.z), as_int(v));
        cell[2 * k + 1] = make_int4(tbeg[t] | (tend[t] << 16), as_int(par.tab4[t][pk.stype[o]].z), t, j);
      }
  }

  std::vector<DevParams> parv(1, par);
  std::vector<float4> ref4((size_t)kLigTypes * kTabCols, make_float4(0.f, 0.f, 0.f, 0.f));
  for (int lt = 0; lt < kLigTypes; ++lt)
    for (int pt = 0; pt < kPadType; ++pt) {
      const bool hb = ep.hdb0[lt][pt] > 0.1f;
      ref4[(size_t)lt * kTabCols + pt] = make_float4(ep.p1a[lt][pt], ep.p2a[lt][pt], hb ? ep.hdb0[lt][pt] : 0.f,
                                                     hb ? ep.hdb1[lt][pt] : 0.f);
    }

  const int nrep = (int)jd.reps.size();
  std::vector<int> run_acc(nrep);
  for (int r = 0; r < nrep; ++r) run_acc[r] = jd.reps[r].is_accept;
  std::vector<RepStats> stats(nrep);
  for (auto &s : stats) {
    std::memset(&s, 0, sizeof(s));
    s.best_step = -1;
  }

  Arena ar;
  const size_t o_par = ar.put(parv), o_lig = ar.put(lig), o_lg = ar.put(lgrp), o_lc = ar.put(jd.lcenter);
  const size_t o_pm = ar.put(pspmask), o_hr = ar.put(ref4);
  const size_t o_pc = ar.put(pcell), o_pcn = ar.put(pcell_cnt), o_ks = ar.put(kslot);
  const size_t o_kde = ar.put(kde), o_mcs = ar.put(mcs), o_tcc = ar.put(jd.tcc), o_psp = ar.put(psp);
  const size_t o_mb = ar.put(jd.minus_beta), o_rep = ar.put(jd.reps), o_acc = ar.put(run_acc), o_st = ar.put(stats);
  size_t o_rec = 0;
  const bool alloc_rec = want_records && rec == nullptr;
  if (alloc_rec) o_rec = ar.take(sizeof(Record) * (size_t)nrep);

  const bool reusing = reuse && reuse->arena && reuse->bytes == ar.off && !alloc_rec;
  if (!reusing && take_injected_alloc_failure())
    return fail(GD_E_NOMEM, "device allocation of %zu B for a job failed (injected by the fail_alloc test hook)", ar.off);
  if (reusing) {
    out.arena = reuse->arena;
    GD_CUDA(cudaMemcpyAsync(out.arena, ar.host.data(), ar.off, cudaMemcpyHostToDevice, st));
  } else if (async) {
    // stream-ordered: no device-wide synchronisation (a pageable copy may wait for `st` only)
    const cudaError_t me = cudaMallocAsync(&out.arena, ar.off, st);
    if (me == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      return fail(GD_E_NOMEM, "cudaMallocAsync of %zu B for a job: out of device memory", ar.off);
    }
    GD_CUDA(me);
    if (alloc_rec) GD_CUDA(cudaMemsetAsync(out.arena, 0, ar.off, st));
    GD_CUDA(cudaMemcpyAsync(out.arena, ar.host.data(), alloc_rec ? o_rec : ar.off, cudaMemcpyHostToDevice, st));
  } else {
    GD_CUDA(cudaMalloc(&out.arena, ar.off));
    if (alloc_rec) GD_CUDA(cudaMemset(out.arena, 0, ar.off));
    GD_CUDA(cudaMemcpy(out.arena, ar.host.data(), alloc_rec ? o_rec : ar.off, cudaMemcpyHostToDevice));
  }
  out.bytes = ar.off;
  out.own_rec = alloc_rec;
  unsigned char *b = (unsigned char *)out.arena;

  DevJob &J = out.dj;
  std::memset(&J, 0, sizeof(J));
  J.natom = L;
  J.nlig = jd.nlig;
  J.lstride = lstride;
  J.lig = (const float4 *)(b + o_lig);
  J.lgrp = (const int2 *)(b + o_lg);
  J.lcenter = (const float *)(b + o_lc);
  J.npoint_pad = P;
  J.nprt = pk.nconf;
  J.pos = pk.pos;
  J.aux = pk.aux;
  J.ncdc = pk.ncdc;
  J.pcenter = pk.center;
  J.psp = (const float *)(b + o_psp);
  J.pspmask = (const uint32_t *)(b + o_pm);
  J.pcell = (const int4 *)(b + o_pc);
  J.pcell_cnt = (const int *)(b + o_pcn);
  J.pcell_stride = cstride;
  J.nkde = (int)kidx.size();
  J.nkslot = nkslot;
  J.kslot = (const int4 *)(b + o_ks);
  J.kde = (const float4 *)(b + o_kde);
  for (int t = 0; t < kLigTypes; ++t) {
    J.kbeg[t] = kbeg[t];
    J.kcnt[t] = kcnt[t];
  }
  J.nmcs = jd.M;
  J.mcs = (const float4 *)(b + o_mcs);
  J.tcc = (const float *)(b + o_tcc);
  J.ntmp = jd.ntmp;
  J.minus_beta = (const float *)(b + o_mb);
  J.par = (const DevParams *)(b + o_par);
  J.ref4 = (const float4 *)(b + o_hr);
  J.nrep = nrep;
  J.rep = (ReplicaMC *)(b + o_rep);
  J.run_acc = (int *)(b + o_acc);
  J.stats = (RepStats *)(b + o_st);
  J.rec = alloc_rec ? (Record *)(b + o_rec) : (want_records ? rec : nullptr);
  J.key0 = (uint32_t)jd.seed;
  J.key1 = (uint32_t)(jd.seed >> 32);
  J.rid_base = jd.rid_base;
  J.nrep_total = jd.nrep_total;
  J.xsweep = -1;
  return GD_OK;
}
}  // namespace

int pack_job(const JobData &jd, const DevPocket &pk, const EnePara &ep, bool want_records, Record *rec,
             DevJobBuf &out, const DevJobBuf *reuse, cudaStream_t st)
{
  return pack_job_impl(jd, pk, ep, want_records, rec, st, false, out, reuse);
}

int pack_job_async(const JobData &jd, const DevPocket &pk, const EnePara &ep, cudaStream_t st, DevJobBuf &out)
{
  return pack_job_impl(jd, pk, ep, false, nullptr, st, true, out);
}

void free_pocket(DevPocket &p)
{
  if (p.arena) cudaFree(p.arena);
  p = DevPocket{};
}

void free_job_async(DevJobBuf &j, cudaStream_t st)
{
  if (j.arena) cudaFreeAsync(j.arena, st);
  j = DevJobBuf{};
}

void free_job(DevJobBuf &j)
{
  if (j.arena) cudaFree(j.arena);
  j = DevJobBuf{};
}

}  // namespace gd
