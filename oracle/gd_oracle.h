/*
 * gd_oracle.h -- FP64 CPU restatement of the GeauxDock Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels.  Only tests/,
 * the smoke check and bench.py's CPU-baseline leg may load liboracle.so.
 *
 * Pinned against (a) the reference's own CPU energy routine compiled from its
 * sources (oracle/_ref/libgdref.so) on synthetic complexes, and (b) the
 * reference's known-answer line for 1a07C1 x 1a07C-1
 * (doc/instructions.txt:186-187, src/common/kernel_print.C:11), and its
 * Philox against the Random123 known-answer vectors
 * (src/module/Random123/examples/kat_vectors:27-29).
 */
#ifndef GD_ORACLE_H
#define GD_ORACLE_H

#include <stdint.h>
#include "gdock_types.h"
#include "gdock.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon et al., SC'11), counter-based. */
void gdo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* 32-bit draw -> float uniform in (0, 1]: ((x >> 8) + 1) * 2^-24. */
float gdo_u01(uint32_t x);

/* Energy of ligand conformation il in protein conformation ip at pose
 * movematrix mm (translation xyz, Euler angles xyz).  e[0..8] are the
 * normalised terms and e[9] the weighted total, as stored in
 * ReplicaMC.energy; raw[0..8] (may be NULL) are the terms before the
 * per-atom division and the a/b normalisation. */
void gdo_energy(const Complex *c, int il, int ip, const float mm[6], double e[10], double raw[9]);

/* The same energy over cap-free dense arrays (gd_pocket_desc_t and
 * gd_job_desc_t layouts): ligand conformation il, protein conformation ip.
 * The ligand atoms are visited in input order for every term. */
void gdo_energy_desc(const gd_pocket_desc_t *pk, const gd_job_desc_t *job, const EnePara *ep, int il, int ip,
                     const float mm[6], double e[10], double raw[9]);
/* n poses (conf[2i], conf[2i+1], mm[6i..]) with OpenMP over poses. */
void gdo_energy_desc_batch(const gd_pocket_desc_t *pk, const gd_job_desc_t *job, const EnePara *ep, int n,
                           const int *conf, const float *mm, double *e, double *raw);

/* Monte Carlo over replicas [rep_begin, rep_end] for steps s1 .. s1+s2max-1,
 * with the draws of the GPU kernels (Philox keyed by seed).  s2max == 1 is the
 * reference's initial-energy call: no move, forced accept.  Records follow
 * src/backend_cpu_mic/kernel_cpp_montecarlo_soa.C:224-231 (record may be
 * NULL).  steps_per_exchange > 0 runs a replica-exchange sweep after every
 * global step s with (s+1) % steps_per_exchange == 0. */
void gdo_montecarlo(Complex *c, Record *record, int s1, int s2max, uint64_t seed, int steps_per_exchange);

/* One replica-exchange sweep with index x over all (ligand conf, protein
 * conf) groups of adjacent temperatures. */
void gdo_exchange(Complex *c, int x, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
