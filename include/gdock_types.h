/*
 * gdock_types.h -- plain-C declarations of the data structures that cross the
 * GeauxDock docking boundary.
 *
 * The layouts below are the wire format of the reference's `Dock(...)` call:
 * a frontend built against the reference fills a `Complex` (a flat POD of
 * 6,583,296 bytes) and a `Record[]` array and hands raw pointers across.  To be
 * a drop-in, every struct here keeps the reference's field order, array caps
 * and 64-byte struct alignment, so `sizeof` and every `offsetof` agree byte for
 * byte.  The static assertions at the bottom pin the sizes measured from the
 * reference headers:
 *   Complex   6,583,296 B   (src/common/geauxdock.h:391-439)
 *   Record       25,664 B   (src/common/geauxdock.h:374-378)
 *   ReplicaMC       128 B   (src/common/geauxdock.h:323-336)
 *   EnePara      18,432 B   (src/common/geauxdock_soa.h:154-187)
 *
 * Capacity constants follow src/common/size.h:21-123.  The device-side layout
 * used by the kernels is separate (packed structure-of-arrays, no caps); these
 * structs exist only at the boundary.
 */
#ifndef GDOCK_TYPES_H
#define GDOCK_TYPES_H

#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GD_ALIGN64 __align__(64)
#else
#define GD_ALIGN64 __attribute__((aligned(64)))
#endif

/* capacity caps (src/common/size.h) */
#define GD_MAX_STR_LENG 256
#define GD_MAXPRO 2048          /* protein effective points            size.h:28 */
#define GD_MAXLIG 64            /* ligand heavy atoms                  size.h:31 */
#define GD_MAX_CONF_PRT 20      /* protein conformations               size.h:34 */
#define GD_MAX_CONF_LIG 64      /* ligand conformations                size.h:37 */
#define GD_MAX_TMP 1024         /* temperatures                        size.h:43 */
#define GD_MAX_REP 16384        /* replicas per Complex                size.h:48 */
#define GD_MAXTP1 31            /* protein point types (30 used)       size.h:62 */
#define GD_MAXTP2 24            /* ligand atom types                   size.h:65 */
#define GD_MAXTP3 50            /* electrostatic point classes         size.h:68 */
#define GD_MAXTP4 20            /* residue types                       size.h:71 */
#define GD_MAXWEI 10            /* energy terms incl. total            size.h:81 */
#define GD_MAXKDE 10240         /* KDE points                          size.h:84 */
#define GD_MAX_MCS_ROW 512      /* MCS template rows                   size.h:87 */
#define GD_MAX_MCS_COL GD_MAXLIG
#define GD_MAXSTRINGLENG 128
#define GD_STEPS_PER_DUMP 200   /* Record capacity per replica         size.h:116 */
#define GD_MCS_INVALID_COORD 0.01234f /* unset MCS template coordinate size.h:107 */

/* energy term indices of ReplicaMC.energy[] (src/common/geauxdock.h:131-147) */
enum {
  GD_E_VDW = 0, GD_E_ELE = 1, GD_E_PMF = 2, GD_E_PSP = 3, GD_E_HDB = 4,
  GD_E_HPC = 5, GD_E_KDE = 6, GD_E_LHM = 7, GD_E_DST = 8, GD_E_TOTAL = 9
};

#ifdef __cplusplus
extern "C" {
#endif

/* Ligand conformation, three coordinate copies (src/common/geauxdock_soa.h:8-44).
 * Copy 2 keeps the input atom order; copy 3 is sorted by atom type; copy 1 is
 * "might be sorted" and unused by the energy routine. */
typedef struct GD_ALIGN64 Ligand {
  float x1[GD_MAXLIG], y1[GD_MAXLIG], z1[GD_MAXLIG];
  int   t1[GD_MAXLIG];
  float c1[GD_MAXLIG];
  float x2[GD_MAXLIG], y2[GD_MAXLIG], z2[GD_MAXLIG];
  int   t2[GD_MAXLIG];
  float c2[GD_MAXLIG];
  float x3[GD_MAXLIG], y3[GD_MAXLIG], z3[GD_MAXLIG];
  int   t3[GD_MAXLIG];
  float c3[GD_MAXLIG];
  int kde_begin_idx[GD_MAXLIG];
  int kde_end_idx[GD_MAXLIG];
  float center[3];      /* ligand centre in the lab frame */
  int lig_natom;
} Ligand;

/* Protein conformation of coarse-grained effective points (geauxdock_soa.h:52-72). */
typedef struct GD_ALIGN64 Protein {
  int   t[GD_MAXPRO];     /* point type 0..29 */
  float x[GD_MAXPRO], y[GD_MAXPRO], z[GD_MAXPRO];
  int   cdc[GD_MAXPRO];   /* hydrophobic-contact flag */
  float hpp[GD_MAXPRO];   /* residue hydrophobicity */
  float ele[GD_MAXPRO];   /* electrostatic point parameter */
  int   c[GD_MAXPRO];     /* point class: 0 CA, 1 peptide plate, 2/3 side chain */
  int   seq3r[GD_MAXPRO]; /* residue serial number, column of Psp */
  float pocket_center[3];
  int prt_npoint;
} Protein;

/* Pocket-specific potential, psp[ligand type][residue serial] (geauxdock_soa.h:77-81). */
typedef struct GD_ALIGN64 Psp {
  float psp[GD_MAXLIG][GD_MAXPRO];
} Psp;

/* KDE points sorted by atom type (geauxdock_soa.h:85-93). */
typedef struct GD_ALIGN64 Kde {
  int   t[GD_MAXKDE];
  float x[GD_MAXKDE], y[GD_MAXKDE], z[GD_MAXKDE];
  int kde_npoint;
} Kde;

/* One MCS template row indexed by ligand atom (geauxdock_soa.h:97-105). */
typedef struct GD_ALIGN64 Mcs {
  float x[GD_MAX_MCS_COL], y[GD_MAX_MCS_COL], z[GD_MAX_MCS_COL];
  int ncol;
  float tcc;
} Mcs;

/* Alternative MCS layouts kept only so that Complex keeps its size
 * (geauxdock_soa.h:109-146); the energy routine reads Mcs only. */
typedef struct GD_ALIGN64 Mcs_R {
  float x[GD_MAX_MCS_COL][GD_MAX_MCS_ROW];
  float y[GD_MAX_MCS_COL][GD_MAX_MCS_ROW];
  float z[GD_MAX_MCS_COL][GD_MAX_MCS_ROW];
  float tcc[GD_MAX_MCS_ROW];
} Mcs_R;

typedef struct GD_ALIGN64 Mcs_ELL {
  int   i[GD_MAX_MCS_ROW][GD_MAX_MCS_COL];
  float x[GD_MAX_MCS_ROW][GD_MAX_MCS_COL];
  float y[GD_MAX_MCS_ROW][GD_MAX_MCS_COL];
  float z[GD_MAX_MCS_ROW][GD_MAX_MCS_COL];
  int ncol[GD_MAX_MCS_ROW];
  float tcc[GD_MAX_MCS_ROW];
} Mcs_ELL;

typedef struct GD_ALIGN64 Mcs_CSR {
  int   idx_col[GD_MAX_MCS_COL * GD_MAX_MCS_ROW];
  int   idx_row[GD_MAX_MCS_COL * GD_MAX_MCS_ROW];
  float x[GD_MAX_MCS_COL * GD_MAX_MCS_ROW];
  float y[GD_MAX_MCS_COL * GD_MAX_MCS_ROW];
  float z[GD_MAX_MCS_COL * GD_MAX_MCS_ROW];
  float tcc[GD_MAX_MCS_ROW];
  int npoint;
} Mcs_CSR;

/* Precomputed force-field parameters, tables indexed [ligand type][point type]
 * (geauxdock_soa.h:154-187; filled by OptimizeEnepara, util_optimize_soa.C:489-540). */
typedef struct GD_ALIGN64 EnePara {
  float p1a[GD_MAXTP2][GD_MAXTP1];   /* 2 eps (sigma lj2)^9 */
  float p2a[GD_MAXTP2][GD_MAXTP1];   /* 3 eps (sigma lj2)^6 */
  float lj0, lj1;
  float el1, el0;
  float a1, b1;                      /* 4-3 el0, 2 el0-3 */
  float pmf0[GD_MAXTP2][GD_MAXTP1];
  float pmf1[GD_MAXTP2][GD_MAXTP1];
  float hdb0[GD_MAXTP2][GD_MAXTP1];
  float hdb1[GD_MAXTP2][GD_MAXTP1];  /* 1/sigma */
  float hpp[GD_MAXTP4];
  float hpl0[GD_MAXTP2], hpl1[GD_MAXTP2], hpl2[GD_MAXTP2];
  float kde2;                        /* -0.5/h^2 */
  float kde3;                        /* (h sqrt(2 pi))^3 */
  float a_para[GD_MAXWEI];           /* normalisation slope */
  float b_para[GD_MAXWEI];           /* normalisation offset */
  float w[GD_MAXWEI];                /* term weights of the total */
} EnePara;

/* Raw force-field parameters as read from the parameter files
 * (src/common/geauxdock.h:279-295); input of OptimizeEnepara. */
typedef struct EnePara0 {
  float vdw[GD_MAXTP1][GD_MAXTP2][2];
  float ele[GD_MAXTP3];
  float pmf[GD_MAXTP1][GD_MAXTP2][2];
  float hpp[GD_MAXTP4];
  float hpl[GD_MAXTP2][2];
  float hdb[GD_MAXTP1][GD_MAXTP2][2];
  float lj[3];
  float el[2];
  float kde;
  float w[GD_MAXWEI];
  float a_para[GD_MAXWEI];
  float b_para[GD_MAXWEI];
} EnePara0;

typedef struct Temp {        /* geauxdock.h:309-314 */
  float t;
  float minus_beta;          /* -1/T */
  int order;
} Temp;

typedef struct GD_ALIGN64 ReplicaMC {   /* geauxdock.h:323-336 */
  int idx_rep, idx_lig, idx_prt, idx_tmp;
  float movematrix[6];       /* translation x y z, rotation x y z */
  float energy[GD_MAXWEI];
  int step;
  int is_accept;
} ReplicaMC;

typedef struct McPara {      /* geauxdock.h:348-358 */
  int steps_total;
  int steps_per_dump;
  int steps_per_exchange;
  float move_scale[6];
  char outputdir[GD_MAXSTRINGLENG];
  char outputfile[GD_MAXSTRINGLENG];
} McPara;

typedef struct Record {      /* geauxdock.h:374-378 */
  ReplicaMC replica[GD_STEPS_PER_DUMP];
  int next_entry;
} Record;

typedef struct ComplexSize { /* geauxdock.h:113-126 */
  int n_lig, n_prt, n_tmp, n_rep;
  int lig_natom, prt_npoint, kde_npoint, mcs_nrow;
} ComplexSize;

typedef struct Complex {     /* geauxdock.h:391-439 */
  Ligand lig[GD_MAX_CONF_LIG];
  Protein prt[GD_MAX_CONF_PRT];
  Psp psp;
  Kde kde;
  Mcs mcs[GD_MAX_MCS_ROW];
  Mcs_R mcs_r;
  Mcs_ELL mcs_ell;
  Mcs_CSR mcs_csr;
  EnePara enepara;
  Temp temp[GD_MAX_TMP];
  ReplicaMC replica[GD_MAX_REP];
  ComplexSize size;
  McPara mcpara;
  char lig_file[GD_MAX_STR_LENG];
  char prt_file[GD_MAX_STR_LENG];
  char lhm_file[GD_MAX_STR_LENG];
  char enepara_file[GD_MAX_STR_LENG];
  char weight_file[GD_MAX_STR_LENG];
  int rep_begin;
  int rep_end;
  int signal;
} Complex;

typedef struct ParaT {       /* geauxdock.h:447-454 */
  int rep_begin, rep_end, n_rep;
  int record_sz;
} ParaT;

#ifdef __cplusplus
}
#endif

#if defined(__cplusplus)
#define GD_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define GD_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
GD_STATIC_ASSERT(sizeof(Complex) == 6583296, "Complex layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(Record) == 25664, "Record layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(ReplicaMC) == 128, "ReplicaMC layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(EnePara) == 18432, "EnePara layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(EnePara0) == 18472, "EnePara0 layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(Ligand) == 4416, "Ligand layout drifted from the reference");
GD_STATIC_ASSERT(sizeof(Protein) == 73792, "Protein layout drifted from the reference");
GD_STATIC_ASSERT(offsetof(Complex, replica) == 4484480, "Complex.replica offset");
GD_STATIC_ASSERT(offsetof(Complex, rep_begin) == 6583236, "Complex.rep_begin offset");
GD_STATIC_ASSERT(offsetof(EnePara, w) == 18336, "EnePara.w offset");

#endif /* GDOCK_TYPES_H */
