/*
 * gd_oracle.c -- FP64 CPU restatement of the GeauxDock Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see gd_oracle.h): the checker for the CUDA
 * kernels, never the thing measured or shipped.
 *
 * Each function follows the reference formulas line by line, in double
 * precision, reading the reference-layout Complex of include/gdock_types.h:
 *   rotation + translation  src/backend_gpu/kernel_cuda_l1_montecarlo.cu:336-380
 *   protein-ligand terms     src/backend_gpu/energy_prt_v1.cu:8-174
 *                            (CPU twin src/backend_cpu_mic/energy_prt_v1.C:5-134)
 *   KDE term                 src/backend_gpu/energy_kde_v1.cu:1-93
 *   MCS term                 src/backend_gpu/energy_mcs_v1.cu:1-45
 *   distance, normalisation  src/backend_gpu/kernel_cuda_l1_montecarlo.cu:404-476
 *   Metropolis + record      src/backend_gpu/kernel_cuda_l1_montecarlo.cu:284-532
 * The draws come from Philox4x32-10 with the counter layout of the GPU
 * kernels, so CPU and GPU trajectories use identical random numbers.
 * Replica exchange has no counterpart in the reference (the fields exist,
 * src/common/geauxdock.h:352, but nothing reads them); it follows the standard
 * parallel-tempering rule between adjacent temperatures of one
 * (ligand conformation, protein conformation) group, the grouping of
 * SetReplica (src/frontend/util.C:371-406).
 */
#include "gd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- Philox -- */

static void mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo)
{
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

void gdo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; ++round) {
    if (round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

float gdo_u01(uint32_t x)
{
  return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

/* Counter layout shared with the GPU kernels: MC draws of global step s of
 * replica r are ctr = {s, r, 0, 0} (move x y z, rot x) and {s, r, 0, 1}
 * (rot y z, accept, spare); exchange draws use domain word 1. */
static void mc_draws(uint64_t seed, int step, int rid, float u[8])
{
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t ctr[4] = {(uint32_t)step, (uint32_t)rid, 0u, 0u};
  uint32_t o[4];
  gdo_philox4x32_10(ctr, key, o);
  for (int i = 0; i < 4; ++i) u[i] = gdo_u01(o[i]);
  ctr[3] = 1u;
  gdo_philox4x32_10(ctr, key, o);
  for (int i = 0; i < 4; ++i) u[4 + i] = gdo_u01(o[i]);
}

/* ---------------------------------------------------------------- energy -- */

static void rotation(const float mm[6], double rot[3][3])
{
  /* kernel_cuda_l1_montecarlo.cu:340-354 */
  const double s1 = sin((double)mm[3]), c1 = cos((double)mm[3]);
  const double s2 = sin((double)mm[4]), c2 = cos((double)mm[4]);
  const double s3 = sin((double)mm[5]), c3 = cos((double)mm[5]);
  rot[0][0] = c1 * c2;
  rot[0][1] = c1 * s2 * s3 - c3 * s1;
  rot[0][2] = s1 * s3 + c1 * c3 * s2;
  rot[1][0] = c2 * s1;
  rot[1][1] = c1 * c3 + s1 * s2 * s3;
  rot[1][2] = c3 * s1 * s2 - c1 * s3;
  rot[2][0] = -s2;
  rot[2][1] = c2 * s3;
  rot[2][2] = c2 * c3;
}

void gdo_energy(const Complex *c, int il, int ip, const float mm[6], double e[10], double raw[9])
{
  const Ligand *lig = &c->lig[il];
  const Protein *prt = &c->prt[ip];
  const Kde *kde = &c->kde;
  const EnePara *ep = &c->enepara;
  const int L = lig->lig_natom;
  const int P = prt->prt_npoint;
  const int K = c->size.kde_npoint;
  const int M = c->size.mcs_nrow;

  double rot[3][3];
  rotation(mm, rot);
  double x2[GD_MAXLIG], y2[GD_MAXLIG], z2[GD_MAXLIG];
  double x3[GD_MAXLIG], y3[GD_MAXLIG], z3[GD_MAXLIG];
  const double tx = (double)mm[0] + (double)lig->center[0];
  const double ty = (double)mm[1] + (double)lig->center[1];
  const double tz = (double)mm[2] + (double)lig->center[2];
  for (int l = 0; l < L; ++l) {
    const double a = lig->x2[l], b = lig->y2[l], d = lig->z2[l];
    x2[l] = rot[0][0] * a + rot[0][1] * b + rot[0][2] * d + tx;
    y2[l] = rot[1][0] * a + rot[1][1] * b + rot[1][2] * d + ty;
    z2[l] = rot[2][0] * a + rot[2][1] * b + rot[2][2] * d + tz;
    const double a3 = lig->x3[l], b3 = lig->y3[l], d3 = lig->z3[l];
    x3[l] = rot[0][0] * a3 + rot[0][1] * b3 + rot[0][2] * d3 + tx;
    y3[l] = rot[1][0] * a3 + rot[1][1] * b3 + rot[1][2] * d3 + ty;
    z3[l] = rot[2][0] * a3 + rot[2][1] * b3 + rot[2][2] * d3 + tz;
  }

  /* protein-ligand pair terms, energy_prt_v1.cu:8-174 */
  double evdw = 0, eele = 0, epmf = 0, epsp = 0, ehdb = 0, ehpc = 0;
  const double lj0 = ep->lj0, lj1 = ep->lj1, el0 = ep->el0, el1 = ep->el1, a1 = ep->a1, b1 = ep->b1;
  for (int l = 0; l < L; ++l) {
    const int lt = lig->t2[l];
    const double lc = lig->c2[l];
    double ehpc1 = 0.0;
    for (int p = 0; p < P; ++p) {
      const int pt = prt->t[p];
      const double dx = x2[l] - (double)prt->x[p];
      const double dy = y2[l] - (double)prt->y[p];
      const double dz = z2[l] - (double)prt->z[p];
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double d4 = d2 * d2;
      const double d = sqrt(d2);

      if (prt->cdc[p] == 1 && d2 <= 81.0) {
        ehpc1 += (double)prt->hpp[p] *
                 (1.0 - (3.5 / 81.0 * d2 - 4.5 / 81.0 / 81.0 * d4 + 2.5 / 81.0 / 81.0 / 81.0 * d4 * d2 -
                         0.5 / 81.0 / 81.0 / 81.0 / 81.0 * d4 * d4));
      }

      const double p1 = (double)ep->p1a[lt][pt] / (d4 * d4 * d);
      const double p2 = (double)ep->p2a[lt][pt] / (d4 * d2);
      const double p4 = p1 * lj0 * (1.0 + lj1 * d2) + 1.0;
      evdw += (p1 - p2) / p4;

      const double s1 = el1 * d;
      const double g1 = (s1 < 1.0) ? (el0 + a1 * s1 * s1 + b1 * s1 * s1 * s1) : (1.0 / s1);
      eele += lc * (double)prt->ele[p] * g1;

      const double dmp = d - (double)ep->pmf0[lt][pt];
      epmf += (double)ep->pmf1[lt][pt] / (1.0 + exp((-0.5 * d + 6.0) * dmp));

      if (prt->c[p] == 2 && dmp <= 0.0) epsp += (double)c->psp.psp[lt][prt->seq3r[p]];

      const double hdb0 = ep->hdb0[lt][pt];
      if (hdb0 > (double)0.1f) {
        const double hdb1 = ep->hdb1[lt][pt];
        const double h3 = (d - hdb0) * hdb1;
        ehdb += hdb1 * exp(-0.5 * h3 * h3);
      }
    }
    const double hpc2 = (ehpc1 - (double)ep->hpl0[lt]) / (double)ep->hpl1[lt];
    ehpc += 0.5 * hpc2 * hpc2 - (double)ep->hpl2[lt];
  }

  /* KDE term, energy_kde_v1.cu:183-274: per atom, mean over same-type points */
  double ekde = 0.0;
  for (int l = 0; l < L; ++l) {
    const int lt = lig->t3[l];
    double s = 0.0;
    int n = 0;
    for (int k = 0; k < K; ++k) {
      if (kde->t[k] != lt) continue;
      const double dx = x3[l] - (double)kde->x[k];
      const double dy = y3[l] - (double)kde->y[k];
      const double dz = z3[l] - (double)kde->z[k];
      s += exp((double)ep->kde2 * (dx * dx + dy * dy + dz * dz));
      ++n;
    }
    if (n != 0) ekde += s / (double)n;
  }

  /* MCS term, energy_mcs_v1.cu:277-320 */
  double elhm = 0.0;
  for (int m = 0; m < M; ++m) {
    const Mcs *row = &c->mcs[m];
    double s = 0.0;
    int n = 0;
    for (int l = 0; l < L; ++l) {
      if (row->x[l] == GD_MCS_INVALID_COORD) continue;
      const double dx = x2[l] - (double)row->x[l];
      const double dy = y2[l] - (double)row->y[l];
      const double dz = z2[l] - (double)row->z[l];
      s += dx * dx + dy * dy + dz * dz;
      ++n;
    }
    elhm += (double)row->tcc * sqrt(s / (double)n);
  }

  /* distance to the pocket centre, kernel_cuda_l1_montecarlo.cu:439-454 */
  double dst = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double t = (double)lig->center[i] + (double)mm[i] - (double)prt->pocket_center[i];
    dst += t * t;
  }

  double r[9];
  r[0] = evdw;
  r[1] = eele;
  r[2] = epmf;
  r[3] = epsp;
  r[4] = ehdb * (-1.0 / sqrt(2.0 * 3.14159265358979323846));
  r[5] = ehpc;
  r[6] = ekde / (double)ep->kde3;
  r[7] = log(elhm / (double)M);
  r[8] = sqrt(dst);
  if (raw)
    for (int i = 0; i < 9; ++i) raw[i] = r[i];

  /* normalisation and weighted total, kernel_cuda_l1_montecarlo.cu:460-476 */
  double tot = 0.0;
  for (int i = 0; i < 9; ++i) {
    double v = r[i];
    if (i < 7) v /= (double)L;
    v = (double)ep->a_para[i] * v + (double)ep->b_para[i];
    e[i] = v;
    tot += (double)ep->w[i] * v;
  }
  e[9] = tot;
}

/* Cap-free twin of gdo_energy over descriptor arrays (the same formulas, the
 * same file:line anchors); psp[lt][seq3r] from the job's [24][psp_ncol] table. */
void gdo_energy_desc(const gd_pocket_desc_t *pk, const gd_job_desc_t *jb, const EnePara *ep, int il, int ip,
                     const float mm[6], double e[10], double raw[9])
{
  const int L = jb->natom, P = pk->npoint, K = jb->nkde, M = jb->nmcs;
  double rot[3][3];
  rotation(mm, rot);
  double *lx = (double *)malloc(sizeof(double) * 3 * (size_t)L);
  const float *src = jb->lig_xyz + (size_t)il * L * 3;
  const float *lcen = jb->lig_center + (size_t)il * 3;
  const double tx = (double)mm[0] + (double)lcen[0];
  const double ty = (double)mm[1] + (double)lcen[1];
  const double tz = (double)mm[2] + (double)lcen[2];
  for (int l = 0; l < L; ++l) {
    const double a = src[3 * l], b = src[3 * l + 1], d = src[3 * l + 2];
    lx[3 * l] = rot[0][0] * a + rot[0][1] * b + rot[0][2] * d + tx;
    lx[3 * l + 1] = rot[1][0] * a + rot[1][1] * b + rot[1][2] * d + ty;
    lx[3 * l + 2] = rot[2][0] * a + rot[2][1] * b + rot[2][2] * d + tz;
  }
  const float *pxyz = pk->xyz + (size_t)ip * P * 3;

  /* protein-ligand pair terms, energy_prt_v1.cu:8-174 */
  double evdw = 0, eele = 0, epmf = 0, epsp = 0, ehdb = 0, ehpc = 0;
  const double lj0 = ep->lj0, lj1 = ep->lj1, el0 = ep->el0, el1 = ep->el1, a1 = ep->a1, b1 = ep->b1;
  for (int l = 0; l < L; ++l) {
    const int lt = jb->lig_type[l];
    const double lc = jb->lig_charge[l];
    double ehpc1 = 0.0;
    for (int p = 0; p < P; ++p) {
      const int pt = pk->type[p];
      const double dx = lx[3 * l] - (double)pxyz[3 * p];
      const double dy = lx[3 * l + 1] - (double)pxyz[3 * p + 1];
      const double dz = lx[3 * l + 2] - (double)pxyz[3 * p + 2];
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double d4 = d2 * d2;
      const double d = sqrt(d2);
      if (pk->cdc[p] == 1 && d2 <= 81.0) {
        ehpc1 += (double)pk->hpp[p] *
                 (1.0 - (3.5 / 81.0 * d2 - 4.5 / 81.0 / 81.0 * d4 + 2.5 / 81.0 / 81.0 / 81.0 * d4 * d2 -
                         0.5 / 81.0 / 81.0 / 81.0 / 81.0 * d4 * d4));
      }
      const double p1 = (double)ep->p1a[lt][pt] / (d4 * d4 * d);
      const double p2 = (double)ep->p2a[lt][pt] / (d4 * d2);
      const double p4 = p1 * lj0 * (1.0 + lj1 * d2) + 1.0;
      evdw += (p1 - p2) / p4;
      const double s1 = el1 * d;
      const double g1 = (s1 < 1.0) ? (el0 + a1 * s1 * s1 + b1 * s1 * s1 * s1) : (1.0 / s1);
      eele += lc * (double)pk->ele[p] * g1;
      const double dmp = d - (double)ep->pmf0[lt][pt];
      epmf += (double)ep->pmf1[lt][pt] / (1.0 + exp((-0.5 * d + 6.0) * dmp));
      if (pk->cls[p] == 2 && dmp <= 0.0) epsp += (double)jb->psp[(size_t)lt * jb->psp_ncol + pk->seq3r[p]];
      const double hdb0 = ep->hdb0[lt][pt];
      if (hdb0 > (double)0.1f) {
        const double hdb1 = ep->hdb1[lt][pt];
        const double h3 = (d - hdb0) * hdb1;
        ehdb += hdb1 * exp(-0.5 * h3 * h3);
      }
    }
    const double hpc2 = (ehpc1 - (double)ep->hpl0[lt]) / (double)ep->hpl1[lt];
    ehpc += 0.5 * hpc2 * hpc2 - (double)ep->hpl2[lt];
  }

  /* KDE term, energy_kde_v1.cu:183-274 */
  double ekde = 0.0;
  for (int l = 0; l < L; ++l) {
    const int lt = jb->lig_type[l];
    double s = 0.0;
    int n = 0;
    for (int k = 0; k < K; ++k) {
      if (jb->kde_type[k] != lt) continue;
      const double dx = lx[3 * l] - (double)jb->kde_xyz[3 * k];
      const double dy = lx[3 * l + 1] - (double)jb->kde_xyz[3 * k + 1];
      const double dz = lx[3 * l + 2] - (double)jb->kde_xyz[3 * k + 2];
      s += exp((double)ep->kde2 * (dx * dx + dy * dy + dz * dz));
      ++n;
    }
    if (n != 0) ekde += s / (double)n;
  }

  /* MCS term, energy_mcs_v1.cu:277-320 */
  double elhm = 0.0;
  for (int m = 0; m < M; ++m) {
    const float *row = jb->mcs_xyz + (size_t)m * L * 3;
    double s = 0.0;
    int n = 0;
    for (int l = 0; l < L; ++l) {
      if (row[3 * l] == GD_MCS_INVALID_COORD) continue;
      const double dx = lx[3 * l] - (double)row[3 * l];
      const double dy = lx[3 * l + 1] - (double)row[3 * l + 1];
      const double dz = lx[3 * l + 2] - (double)row[3 * l + 2];
      s += dx * dx + dy * dy + dz * dz;
      ++n;
    }
    elhm += (double)jb->mcs_tcc[m] * sqrt(s / (double)n);
  }

  /* distance to the pocket centre, kernel_cuda_l1_montecarlo.cu:439-454 */
  double dst = 0.0;
  for (int i = 0; i < 3; ++i) {
    const double t = (double)lcen[i] + (double)mm[i] - (double)pk->center[3 * ip + i];
    dst += t * t;
  }
  free(lx);

  double r[9];
  r[0] = evdw;
  r[1] = eele;
  r[2] = epmf;
  r[3] = epsp;
  r[4] = ehdb * (-1.0 / sqrt(2.0 * 3.14159265358979323846));
  r[5] = ehpc;
  r[6] = ekde / (double)ep->kde3;
  r[7] = log(elhm / (double)M);
  r[8] = sqrt(dst);
  if (raw)
    for (int i = 0; i < 9; ++i) raw[i] = r[i];
  double tot = 0.0;
  for (int i = 0; i < 9; ++i) {
    double v = r[i];
    if (i < 7) v /= (double)L;
    v = (double)ep->a_para[i] * v + (double)ep->b_para[i];
    e[i] = v;
    tot += (double)ep->w[i] * v;
  }
  e[9] = tot;
}

void gdo_energy_desc_batch(const gd_pocket_desc_t *pk, const gd_job_desc_t *job, const EnePara *ep, int n,
                           const int *conf, const float *mm, double *e, double *raw)
{
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n; ++i)
    gdo_energy_desc(pk, job, ep, conf[2 * i], conf[2 * i + 1], mm + 6 * (size_t)i, e + 10 * (size_t)i,
                    raw ? raw + 9 * (size_t)i : NULL);
}

/* ----------------------------------------------------------- Monte Carlo -- */

static int replica_step(Complex *c, Record *record, int r, int s, int s2max, uint64_t seed, int *run_acc)
{
  ReplicaMC *rep = &c->replica[r];
  const int rr = r - c->rep_begin;
  if (*run_acc == 1) {
    /* record the old state, kernel_cuda_l1_montecarlo.cu:290-297 */
    rep->step = s;
    if (record) {
      const int ne = record[rr].next_entry;
      record[rr].replica[ne] = *rep;
      record[rr].next_entry = ne + 1;
    }
  }
  float u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (s2max != 1) mc_draws(seed, s, r, u);
  float mm[6];
  for (int i = 0; i < 6; ++i) mm[i] = fmaf(c->mcpara.move_scale[i], u[i], rep->movematrix[i]);

  double e[10];
  gdo_energy(c, rep->idx_lig, rep->idx_prt, mm, e, NULL);
  float ef[10];
  for (int i = 0; i < 10; ++i) ef[i] = (float)e[i];

  int accept;
  if (s2max == 1) {
    accept = 1; /* initial evaluation is always accepted */
  } else {
    const double lr = ((double)ef[9] - (double)rep->energy[9]) * (double)c->temp[rep->idx_tmp].minus_beta;
    accept = log((double)u[6]) < lr;
  }
  if (accept) {
    for (int i = 0; i < 10; ++i) rep->energy[i] = ef[i];
    for (int i = 0; i < 6; ++i) rep->movematrix[i] = mm[i];
  }
  *run_acc = accept;
  return accept;
}

static void exchange_sweep(Complex *c, int x, uint64_t seed, int *run_acc)
{
  const int n_lig = c->size.n_lig, n_prt = c->size.n_prt, n_tmp = c->size.n_tmp;
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  for (int p = 0; p < n_prt; ++p) {
    for (int l = 0; l < n_lig; ++l) {
      const int g = p * n_lig + l;
      for (int t = (x & 1); t + 1 < n_tmp; t += 2) {
        const int ra = n_tmp * n_lig * p + n_lig * t + l;
        const int rb = ra + n_lig;
        if (ra < c->rep_begin || rb > c->rep_end) continue;
        ReplicaMC *a = &c->replica[ra], *b = &c->replica[rb];
        const uint32_t ctr[4] = {(uint32_t)x, (uint32_t)g, 1u, (uint32_t)t};
        uint32_t o[4];
        gdo_philox4x32_10(ctr, key, o);
        const double u = (double)gdo_u01(o[0]);
        /* beta = -minus_beta; accept with min(1, exp((beta_a - beta_b)(E_a - E_b))) */
        const double ba = -(double)c->temp[t].minus_beta, bb = -(double)c->temp[t + 1].minus_beta;
        const double lr = (ba - bb) * ((double)a->energy[9] - (double)b->energy[9]);
        if (log(u) < lr) {
          float tmp[10];
          memcpy(tmp, a->energy, sizeof(tmp));
          memcpy(a->energy, b->energy, sizeof(tmp));
          memcpy(b->energy, tmp, sizeof(tmp));
          float tm[6];
          memcpy(tm, a->movematrix, sizeof(tm));
          memcpy(a->movematrix, b->movematrix, sizeof(tm));
          memcpy(b->movematrix, tm, sizeof(tm));
          run_acc[ra - c->rep_begin] = 1;
          run_acc[rb - c->rep_begin] = 1;
        }
      }
    }
  }
}

void gdo_exchange(Complex *c, int x, uint64_t seed)
{
  const int n = c->rep_end - c->rep_begin + 1;
  int *run_acc = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) run_acc[i] = c->replica[c->rep_begin + i].is_accept;
  exchange_sweep(c, x, seed, run_acc);
  for (int i = 0; i < n; ++i) c->replica[c->rep_begin + i].is_accept = run_acc[i];
  free(run_acc);
}

void gdo_montecarlo(Complex *c, Record *record, int s1, int s2max, uint64_t seed, int steps_per_exchange)
{
  const int n = c->rep_end - c->rep_begin + 1;
  if (n <= 0) return;
  int *run_acc = (int *)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    run_acc[i] = c->replica[c->rep_begin + i].is_accept;
    if (record) record[i].next_entry = 0;
  }
  int s2 = 0;
  while (s2 < s2max) {
    /* run up to the next exchange boundary, all replicas in lock step */
    int end = s2max;
    if (steps_per_exchange > 0 && s2max != 1) {
      const int s = s1 + s2;
      const int next = (s / steps_per_exchange + 1) * steps_per_exchange; /* first step index after the sweep */
      if (next - s1 < end) end = next - s1;
    }
    for (int r = c->rep_begin; r <= c->rep_end; ++r)
      for (int k = s2; k < end; ++k) replica_step(c, record, r, s1 + k, s2max, seed, &run_acc[r - c->rep_begin]);
    if (steps_per_exchange > 0 && s2max != 1 && ((s1 + end) % steps_per_exchange) == 0)
      exchange_sweep(c, (s1 + end) / steps_per_exchange - 1, seed, run_acc);
    s2 = end;
  }
  for (int i = 0; i < n; ++i) c->replica[c->rep_begin + i].is_accept = run_acc[i];
  free(run_acc);
}
