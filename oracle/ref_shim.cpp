// ref_shim.cpp -- C entry points around the reference's own CPU docking code.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's unmodified CPU sources (the recipe is oracle/Makefile) into
// oracle/_ref/libgdref.so.  Only the tests, the smoke check and the CPU
// baseline arm of bench.py load that library, and only as a checker or as the
// timed reference; the product path never touches it.
//
// What it exposes:
//   * the reference's public CPU entry point Dock(Complex*, Record*)
//     (src/backend_cpu_mic/backend_cpu_mic.C:33-127) and its Monte Carlo
//     kernel MonteCarlo_d (src/backend_cpu_mic/kernel_cpp_montecarlo_soa.C:32-418),
//     which with s2max == 1 evaluates the energy of each replica's stored pose
//     and force-accepts it (:248, :384);
//   * the reference frontend run for one ligand and one protein, in the order
//     of src/frontend/server1.C:52-217, used to pin the known-answer line of
//     doc/instructions.txt:186-187 on the shipped 1a07C1 x 1a07C-1 example;
//   * the parameter-file loaders (src/frontend/load.C:1189-1507) and
//     OptimizeEnepara (src/frontend/util_optimize_soa.C:489-540).
//
// The reference structs are used here through the reference's own headers; the
// exported functions take void* so that callers can pass the byte-compatible
// structs of include/gdock_types.h.

#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <omp.h>

#include <size.h>
#include <toggle.h>
#include <geauxdock.h>
#include <util.h>
#include <util_optimize.h>
#include <load.h>

// The reference backend: defines Dock() and the static MonteCarlo_d().
#include <backend_cpu_mic.C>

// loadLigand calls the Fortran superposition routine u3b_ (src/frontend/rmsd.f,
// Kabsch's algorithm) only to drop near-duplicate conformers
// (src/frontend/load.C:421-428); gfortran is absent, so this restates what it
// returns there: *rms = the weighted sum of squared deviations after the
// optimal rotation and translation of x onto y.  Kabsch (Acta Cryst. A32, 922
// (1976); A34, 827 (1978)): with the weighted centred correlation R = sum w a b^T,
// E = sum w (|a|^2 + |b|^2) - 2 (s1 + s2 + sign(det R) s3), s_i the singular
// values of R (square roots of the eigenvalues of R^T R, here by Jacobi
// rotations).  u and t are left as the identity and zero (the caller reads
// only rms).
extern "C" void u3b_(float (*w)[MAXLIG], float (*x)[MAXLIG][3], float (*y)[MAXLIG][3], int *n, int *mode,
                     float *rms, float (*u)[3][3], float (*t)[3], int *ier)
{
  (void)mode;
  const int m = *n;
  double W = 0, xc[3] = {0, 0, 0}, yc[3] = {0, 0, 0};
  for (int i = 0; i < m; ++i) {
    W += (*w)[i];
    for (int k = 0; k < 3; ++k) {
      xc[k] += (*w)[i] * (*x)[i][k];
      yc[k] += (*w)[i] * (*y)[i][k];
    }
  }
  for (int k = 0; k < 3; ++k) {
    xc[k] /= W;
    yc[k] /= W;
  }
  double R[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e0 = 0;
  for (int i = 0; i < m; ++i) {
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = (*x)[i][k] - xc[k];
      b[k] = (*y)[i][k] - yc[k];
      e0 += (*w)[i] * (a[k] * a[k] + b[k] * b[k]);
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) R[r][c] += (*w)[i] * a[r] * b[c];
  }
  const double det = R[0][0] * (R[1][1] * R[2][2] - R[1][2] * R[2][1]) -
                     R[0][1] * (R[1][0] * R[2][2] - R[1][2] * R[2][0]) +
                     R[0][2] * (R[1][0] * R[2][1] - R[1][1] * R[2][0]);
  double M[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) M[r][c] = R[0][r] * R[0][c] + R[1][r] * R[1][c] + R[2][r] * R[2][c];
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = M[0][1] * M[0][1] + M[0][2] * M[0][2] + M[1][2] * M[1][2];
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (M[p][q] == 0.0) continue;
        const double th = 0.5 * std::atan2(2.0 * M[p][q], M[q][q] - M[p][p]);
        const double c = std::cos(th), s = std::sin(th);
        for (int k = 0; k < 3; ++k) {
          const double kp = M[k][p], kq = M[k][q];
          M[k][p] = c * kp - s * kq;
          M[k][q] = s * kp + c * kq;
        }
        for (int k = 0; k < 3; ++k) {
          const double pk = M[p][k], qk = M[q][k];
          M[p][k] = c * pk - s * qk;
          M[q][k] = s * pk + c * qk;
        }
      }
  }
  double sv[3] = {std::sqrt(std::max(M[0][0], 0.0)), std::sqrt(std::max(M[1][1], 0.0)),
                  std::sqrt(std::max(M[2][2], 0.0))};
  std::sort(sv, sv + 3);
  const double e = e0 - 2.0 * (sv[2] + sv[1] + (det < 0 ? -sv[0] : sv[0]));
  *rms = (float)std::max(e, 0.0);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) (*u)[i][j] = (i == j) ? 1.0f : 0.0f;
    (*t)[i] = 0.0f;
  }
  *ier = 0;
}

extern "C" {

size_t gdref_sizeof(const char *name)
{
  const std::string n(name);
  if (n == "Complex") return sizeof(Complex);
  if (n == "Record") return sizeof(Record);
  if (n == "ReplicaMC") return sizeof(ReplicaMC);
  if (n == "EnePara") return sizeof(EnePara);
  if (n == "EnePara0") return sizeof(EnePara0);
  return 0;
}

void gdref_set_threads(int n)
{
  if (n > 0) omp_set_num_threads(n);
}

int gdref_max_threads(void) { return omp_get_max_threads(); }

// The reference's public CPU entry point (prints its own report to stdout).
void gdref_dock(void *complex, void *record)
{
  Dock((Complex *)complex, (Record *)record);
}

// The reference Monte Carlo kernel over replicas [rep_begin, rep_end].
void gdref_montecarlo(void *complex, void *record, int s1, int s2max)
{
  MonteCarlo_d((Complex *)complex, (Record *)record, s1, s2max);
}

// Parameter files -> EnePara0 (raw) and EnePara (precomputed), reference order:
// loadEnePara, loadWeight, loadNorPara, OptimizeEnepara (server1.C:71-78).
// The raw struct is zero-filled first; the reference leaves it uninitialised.
void gdref_load_enepara(const char *paras, const char *weight, const char *nor_a, const char *nor_b,
                        void *enepara0_out, void *enepara_out)
{
  EnePara0 *e0 = (EnePara0 *)enepara0_out;
  std::memset(e0, 0, sizeof(EnePara0));
  EneParaFile ef; ef.path = paras;
  WeightFile wf; wf.path = weight;
  NorParaFile nf; nf.path_a = nor_a; nf.path_b = nor_b;
  loadEnePara(&ef, e0);
  loadWeight(&wf, e0);
  loadNorPara(&nf, e0);
  std::memset(enepara_out, 0, sizeof(EnePara));
  OptimizeEnepara(e0, (EnePara *)enepara_out);
}

// The reference's OptimizeEnepara (util_optimize_soa.C:489-540) on a raw
// parameter set: the precomputed tables a Complex carries.
void gdref_optimize_enepara(const void *enepara0, void *enepara_out)
{
  std::memset(enepara_out, 0, sizeof(EnePara));
  OptimizeEnepara((EnePara0 *)enepara0, (EnePara *)enepara_out);
}

// One ligand (.sdf + .ff) against one protein (.pdb), assembled into a Complex
// exactly as src/frontend/server1.C:52-217 does for complex i.  Returns the
// number of replicas.
int gdref_load_complex(const char *ligand_id, const char *sdf, const char *ff, const char *pdb,
                       const char *paras, const char *weight, const char *nor_a, const char *nor_b,
                       int num_temp, float floor_temp, float ceiling_temp, float ts, float rs,
                       int steps_total, int steps_per_dump, void *complex_out)
{
  Complex *cc = (Complex *)complex_out;
  std::memset(cc, 0, sizeof(Complex));

  LigandFile lf;
  lf.path = sdf;
  lf.molid = "MOLID";
  LhmFile hf;
  hf.path = ff;
  hf.ligand_id = ligand_id;

  // value-initialised: loadLigand accumulates the centre into coord_orig.center
  // and pocket_center (load.C:285-288) and relies on them starting at zero.
  Ligand0 *lig0 = new Ligand0[MAX_CONF_LIG]();
  Psp0 *psp0 = (Psp0 *)std::calloc(1, sizeof(Psp0));
  // loadLHM counts KDE points per type with kde->pns[getLigCode(t)]++
  // (load.C:1106); an unknown type gives code BADKDE = 50 (data.C:582-584) and pns holds
  // MAXTP2 = 24 entries (geauxdock.h:252), so the count lands past the struct.
  // The slack keeps that stray increment inside this allocation; without it the
  // increment hits whatever the heap put next (here, mcs0[0].x[23]).
  Kde0 *kde0 = (Kde0 *)std::calloc(1, sizeof(Kde0) + 64 * sizeof(int));
  Mcs0 *mcs0 = (Mcs0 *)std::calloc(MAX_MCS_ROW, sizeof(Mcs0));
  Ligand *ligs = (Ligand *)std::calloc(MAX_CONF_LIG, sizeof(Ligand));
  Psp *psp = (Psp *)std::calloc(1, sizeof(Psp));
  Kde *kde = (Kde *)std::calloc(1, sizeof(Kde));
  Mcs *mcs = (Mcs *)std::calloc(MAX_MCS_ROW, sizeof(Mcs));
  Mcs_R *mcs_r = (Mcs_R *)std::calloc(1, sizeof(Mcs_R));
  Mcs_ELL *mcs_ell = (Mcs_ELL *)std::calloc(1, sizeof(Mcs_ELL));
  Mcs_CSR *mcs_csr = (Mcs_CSR *)std::calloc(1, sizeof(Mcs_CSR));

  loadLigand(&lf, lig0);
  loadLHM(&hf, psp0, kde0, mcs0);
  OptimizeKde(kde0, kde);
  OptimizeLigand(lig0, kde, ligs, lf.conf_total);
  OptimizePsp(psp0, psp);
  OptimizeMcs(mcs0, mcs, mcs_r, mcs_ell, mcs_csr, hf.mcs_nrow);

  EnePara0 *enepara0 = (EnePara0 *)std::calloc(1, sizeof(EnePara0));
  EnePara *enepara = (EnePara *)std::calloc(1, sizeof(EnePara));
  gdref_load_enepara(paras, weight, nor_a, nor_b, enepara0, enepara);

  ProteinFile pf;
  pf.path = pdb;
  Protein0 *prt0 = (Protein0 *)std::calloc(MAX_CONF_PRT, sizeof(Protein0));
  Protein *prt = (Protein *)std::calloc(MAX_CONF_PRT, sizeof(Protein));
  loadProtein(&pf, prt0);
  SetPocketCenter(prt, lig0[0].pocket_center[0], lig0[0].pocket_center[1], lig0[0].pocket_center[2],
                  pf.conf_total);
  OptimizeProtein(prt0, prt, enepara0, pf.conf_total);

  ComplexSize sz;
  sz.n_prt = pf.conf_total;
  sz.n_lig = lf.conf_total;
  sz.n_tmp = num_temp;
  sz.n_rep = sz.n_lig * sz.n_prt * sz.n_tmp;
  sz.lig_natom = lf.lig_natom;
  sz.prt_npoint = pf.prt_npoint;
  sz.kde_npoint = kde0->kde_npoint;
  sz.mcs_nrow = hf.mcs_nrow;

  ExchgPara ex;
  ex.floor_temp = floor_temp;
  ex.ceiling_temp = ceiling_temp;
  ex.num_temp = num_temp;
  Temp *temp = (Temp *)std::calloc(MAX_TMP, sizeof(Temp));
  ReplicaMC *replica = (ReplicaMC *)std::calloc(MAX_REP, sizeof(ReplicaMC));
  SetTemperature(temp, &ex);
  SetReplica(replica, sz);

  McPara mp;
  std::memset(&mp, 0, sizeof(mp));
  mp.steps_total = steps_total;
  mp.steps_per_dump = steps_per_dump;
  for (int i = 0; i < 3; ++i) mp.move_scale[i] = ts;
  for (int i = 3; i < 6; ++i) mp.move_scale[i] = rs;

  cc->size = sz;
  cc->mcpara = mp;
  cc->psp = *psp;
  cc->kde = *kde;
  cc->enepara = *enepara;
  for (int j = 0; j < sz.n_lig; ++j) cc->lig[j] = ligs[j];
  for (int j = 0; j < sz.n_prt; ++j) cc->prt[j] = prt[j];
  for (int j = 0; j < sz.mcs_nrow; ++j) cc->mcs[j] = mcs[j];
  cc->mcs_r = *mcs_r;
  cc->mcs_ell = *mcs_ell;
  cc->mcs_csr = *mcs_csr;
  for (int j = 0; j < sz.n_tmp; ++j) cc->temp[j] = temp[j];
  for (int j = 0; j < sz.n_rep; ++j) cc->replica[j] = replica[j];
  cc->rep_begin = 0;
  cc->rep_end = sz.n_rep - 1;

  delete[] lig0;
  std::free(psp0); std::free(kde0); std::free(mcs0); std::free(ligs); std::free(psp); std::free(kde);
  std::free(mcs); std::free(mcs_r); std::free(mcs_ell); std::free(mcs_csr); std::free(enepara0);
  std::free(enepara); std::free(prt0); std::free(prt); std::free(temp); std::free(replica);
  return sz.n_rep;
}

}  // extern "C"
