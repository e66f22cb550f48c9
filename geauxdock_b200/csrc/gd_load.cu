// gd_load.cu -- the reference frontend's input path for one docking job:
// ligand .sdf with its conformer ensemble, .ff file (KDE points, pocket-specific
// potential, MCS templates) and protein .pdb models, into a reference-layout
// Complex as the GPU frontend builds it (src/frontend/load.C, data.C,
// util_optimize_soa.C, util.C).  Host code only.
//
// Parsing follows the reference's rules, quirks included, because the files
// are only meaningful under them: fixed columns of the SDF atom block and the
// PDB ATOM records, atof-then-float conversion, the first "$$$$" molecule,
// PDB models delimited by ENDMDL, residues matched by serial number only,
// every MCS line counted as a row.  Conformers within 0.1 A RMSD of the native
// pose (after optimal superposition) are dropped, as the reference does with
// the Fortran routine u3b (src/frontend/rmsd.f), here by Horn's closed-form
// quaternion solution (J. Opt. Soc. Am. A 4, 629 (1987)).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <initializer_list>
#include <sstream>
#include <string>
#include <vector>

#include "gd_internal.h"
#include "gd_pack.h"
#include "gdock.h"

using namespace gd;

namespace {

constexpr int kBadKde = 50;  // getLigCode's code for an unknown type (size.h:101)

int read_lines(const char *path, std::vector<std::string> &out)
{
  if (!path) return fail(GD_E_INVALID, "null path");
  std::ifstream f(path);
  if (!f.is_open()) return fail(GD_E_INVALID, "cannot open %s", path);
  std::string s;
  while (std::getline(f, s)) out.push_back(s);
  return GD_OK;
}

std::vector<std::string> tokens(const std::string &s)
{
  std::vector<std::string> t;
  std::istringstream in(s);
  std::string w;
  while (in >> w) t.push_back(w);
  return t;
}

float to_f(const std::string &s) { return (float)std::atof(s.c_str()); }  // atof, then float

std::string field(const std::string &s, size_t pos, size_t n) { return pos <= s.size() ? s.substr(pos, n) : ""; }

// SYBYL atom type -> ligand type code (data.C:531-586)
int lig_code(const std::string &n)
{
  static const char *names[24] = {"Br",  "C.1",  "C.2",  "C.3",   "C.ar",  "C.cat", "Cl",  "F",
                                  "I",   "N.1",  "N.2",  "N.3",   "N.4",   "N.am",  "N.ar", "N.pl3",
                                  "O.2", "O.3",  "O.co2", "P.3",  "S.2",   "S.3",   "S.O", "S.O2"};
  for (int i = 0; i < 24; ++i)
    if (n == names[i]) return i;
  return kBadKde;
}

// residue name -> residue code (data.C:238-286); -1 for an unknown name
int res_code(const std::string &n)
{
  static const char *names[20] = {"ALA", "ARG", "CYS", "PRO", "LEU", "ILE", "GLU", "HIS", "TRP", "THR",
                                  "MET", "ASP", "GLY", "PHE", "LYS", "GLN", "SER", "ASN", "TYR", "VAL"};
  for (int i = 0; i < 20; ++i)
    if (n == names[i]) return i;
  return -1;
}

// Side-chain points of a residue: (point type, class) pairs (load.C:533-604).
int side_chain(int res, int out[2][2])
{
  static const int tab[20][4] = {{2, 2, -1, -1},  {21, 2, 22, 3}, {3, 2, -1, -1},  {18, 2, -1, -1}, {14, 2, -1, -1},
                                 {11, 2, -1, -1}, {5, 2, 6, 3},   {9, 2, 10, 3},   {26, 2, 27, 3},  {24, 2, -1, -1},
                                 {15, 2, 16, 3},  {4, 2, -1, -1}, {-1, -1, -1, -1}, {7, 2, 8, 3},   {12, 2, 13, 3},
                                 {19, 2, 20, 3},  {23, 2, -1, -1}, {17, 2, -1, -1}, {28, 2, 29, 3}, {25, 2, -1, -1}};
  int n = 0;
  for (int k = 0; k < 2; ++k)
    if (tab[res][2 * k] >= 0) {
      out[n][0] = tab[res][2 * k];
      out[n][1] = tab[res][2 * k + 1];
      ++n;
    }
  return n;
}

// Weighted sum of squared deviations after the optimal rigid superposition of
// `mob` onto `ref` (unit weights): sum |x - xbar|^2 + |y - ybar|^2 - 2 lambda_max
// of Horn's 4x4 matrix, lambda_max by cyclic Jacobi rotations.
double superposed_sq_dev(const float (*mob)[3], const float (*ref)[3], int n)
{
  double mc[3] = {0, 0, 0}, rc[3] = {0, 0, 0};
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      mc[k] += mob[i][k];
      rc[k] += ref[i][k];
    }
  for (int k = 0; k < 3; ++k) {
    mc[k] /= n;
    rc[k] /= n;
  }
  double S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, g = 0.0;
  for (int i = 0; i < n; ++i) {
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = mob[i][k] - mc[k];
      b[k] = ref[i][k] - rc[k];
      g += a[k] * a[k] + b[k] * b[k];
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) S[r][c] += a[r] * b[c];
  }
  const double xx = S[0][0], xy = S[0][1], xz = S[0][2], yx = S[1][0], yy = S[1][1], yz = S[1][2], zx = S[2][0],
               zy = S[2][1], zz = S[2][2];
  double N[4][4] = {{xx + yy + zz, yz - zy, zx - xz, xy - yx},
                    {yz - zy, xx - yy - zz, xy + yx, zx + xz},
                    {zx - xz, xy + yx, -xx + yy - zz, yz + zy},
                    {xy - yx, zx + xz, yz + zy, -xx - yy + zz}};
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) off += N[p][q] * N[p][q];
    if (off < 1e-30) break;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) {
        if (N[p][q] == 0.0) continue;
        const double th = (N[q][q] - N[p][p]) / (2.0 * N[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 4; ++k) {  // N <- J^T N J
          const double kp = N[k][p], kq = N[k][q];
          N[k][p] = c * kp - s * kq;
          N[k][q] = s * kp + c * kq;
        }
        for (int k = 0; k < 4; ++k) {
          const double pk = N[p][k], qk = N[q][k];
          N[p][k] = c * pk - s * qk;
          N[q][k] = s * pk + c * qk;
        }
      }
  }
  const double lmax = std::max(std::max(N[0][0], N[1][1]), std::max(N[2][2], N[3][3]));
  return std::max(0.0, g - 2.0 * lmax);
}

struct SortKey {
  int id;
  double val;
};
// the reference orders points with std::sort on (index, value) records and a
// strict value comparison (util_optimize_soa.C:19-23); the same call gives
// the same order for equal values
std::vector<int> order_by(const std::vector<double> &v)
{
  std::vector<SortKey> k(v.size());
  for (size_t i = 0; i < v.size(); ++i) k[i] = SortKey{(int)i, v[i]};
  std::sort(k.begin(), k.end(), [](const SortKey &a, const SortKey &b) { return a.val < b.val; });
  std::vector<int> o(v.size());
  for (size_t i = 0; i < v.size(); ++i) o[i] = k[i].id;
  return o;
}

struct LigandIn {
  int natom = 0, nconf = 0;
  std::vector<int> type;
  std::vector<float> charge;
  std::vector<float> xyz;  // [nconf][natom][3], centred per conformer
  float center[3] = {0, 0, 0};
};

// loadLigand, load.C:139-456
int read_sdf(const char *path, const char *molid, LigandIn &L)
{
  std::vector<std::string> lines;
  GD_TRY(read_lines(path, lines));
  size_t end = 0;
  while (end < lines.size() && lines[end] != "$$$$") ++end;
  if (end == lines.size() || end + 1 <= 10) return fail(GD_E_INVALID, "%s: no molecule block ending in $$$$", path);
  auto line = [&](size_t i) -> const std::string & {
    static const std::string empty;
    return i < end ? lines[i] : empty;
  };
  const int natom = std::atoi(field(line(3), 0, 3).c_str());
  const int nbond = std::atoi(field(line(3), 3, 3).c_str());
  if (natom < 1 || natom > GD_MAXLIG) return fail(GD_E_CAPACITY, "%s: %d atoms (1..%d)", path, natom, GD_MAXLIG);
  if (nbond < 0 || (size_t)(4 + natom + nbond) > end) return fail(GD_E_INVALID, "%s: truncated atom/bond block", path);
  std::vector<int> type(GD_MAXLIG, 0);
  std::vector<float> charge(GD_MAXLIG, 0.f);
  std::vector<std::vector<float>> raw;  // ensemble coordinates
  const std::string mol = molid ? molid : "MOLID";
  static const char *skip[] = {"SMILES_CANONICAL", "OB_MW", "OB_logP", "OB_PSA", "OB_MR", "MCT_HBD", "MCT_HBA"};
  for (size_t i = 4 + natom + nbond; i < end; ++i) {
    const std::string &s = line(i);
    if (s.find(mol) != std::string::npos) continue;
    bool meta = false;
    for (const char *k : skip) meta = meta || s.find(k) != std::string::npos;
    if (meta) continue;
    if (s.find("OB_ATOM_TYPES") != std::string::npos) {
      const auto t = tokens(line(i + 1));
      for (size_t a = 0; a < t.size() && a < (size_t)GD_MAXLIG; ++a) type[a] = lig_code(t[a]);
    } else if (s.find("OB_ATOMIC_CHARGES") != std::string::npos) {
      const auto t = tokens(line(i + 1));
      for (size_t a = 0; a < t.size() && a < (size_t)GD_MAXLIG; ++a) charge[a] = to_f(t[a]);
    } else if (s.find("ENSEMBLE_COORDS") != std::string::npos) {
      while (line(++i).size() && raw.size() < (size_t)GD_MAX_CONF_LIG) {
        std::vector<float> c((size_t)GD_MAXLIG * 3, 0.f);
        const auto t = tokens(line(i));
        for (size_t k = 0; k < t.size() && k < c.size(); ++k) c[k] = to_f(t[k]);
        raw.push_back(c);
      }
    }
  }
  // native pose from the atom block, centred (float sums as the reference)
  std::vector<float> nat((size_t)natom * 3);
  for (int a = 0; a < natom; ++a) {
    const std::string &s = line(a + 4);
    nat[3 * a] = to_f(field(s, 0, 10));
    nat[3 * a + 1] = to_f(field(s, 10, 10));
    nat[3 * a + 2] = to_f(field(s, 20, 10));
    for (int k = 0; k < 3; ++k) L.center[k] += nat[3 * a + k];
  }
  for (int k = 0; k < 3; ++k) L.center[k] /= (float)natom;
  for (int a = 0; a < natom; ++a)
    for (int k = 0; k < 3; ++k) nat[3 * a + k] -= L.center[k];
  L.natom = natom;
  L.type.assign(type.begin(), type.begin() + natom);
  L.charge.assign(charge.begin(), charge.begin() + natom);
  L.xyz = nat;
  L.nconf = 1;
  // the ensemble, each conformer centred, near-duplicates of the native pose dropped
  for (const auto &c : raw) {
    std::vector<float> mob((size_t)natom * 3);
    float cen[3] = {0, 0, 0};
    for (int a = 0; a < natom; ++a)
      for (int k = 0; k < 3; ++k) cen[k] += c[3 * a + k];
    for (int k = 0; k < 3; ++k) cen[k] /= (float)natom;
    for (int a = 0; a < natom; ++a)
      for (int k = 0; k < 3; ++k) mob[3 * a + k] = c[3 * a + k] - cen[k];
    const float e = (float)superposed_sq_dev(reinterpret_cast<const float(*)[3]>(mob.data()),
                                             reinterpret_cast<const float(*)[3]>(nat.data()), natom);
    const float rms = std::sqrt(e / (float)natom);
    if (rms > 0.1f) {
      L.xyz.insert(L.xyz.end(), mob.begin(), mob.end());
      ++L.nconf;
    }
    if (L.nconf >= GD_MAX_CONF_LIG) break;
  }
  return GD_OK;
}

struct LhmIn {
  std::vector<int> kt;
  std::vector<float> kxyz;
  std::vector<float> psp;  // [MAXPRO][MAXLIG] as read (residue serial, ligand type)
  int nrow = 0;
  std::vector<Mcs> rows;
  std::vector<std::vector<int>> cols;       // column index per entry
  std::vector<std::vector<float>> entries;  // x y z per entry
};

// loadLHM, load.C:1055-1186
int read_ff(const char *path, const char *ligand_id, LhmIn &H)
{
  std::vector<std::string> lines;
  GD_TRY(read_lines(path, lines));
  H.psp.assign((size_t)GD_MAXPRO * GD_MAXLIG, 0.f);
  const std::string id = ligand_id ? ligand_id : "";
  for (const std::string &s : lines) {
    if (s.size() <= 3) continue;
    const std::string tag = s.substr(0, 3);
    const auto t = tokens(s);
    if (tag == "KDE") {
      if (t.size() < 5) return fail(GD_E_INVALID, "%s: short KDE line", path);
      if ((int)H.kt.size() >= GD_MAXKDE) return fail(GD_E_CAPACITY, "%s: more than %d KDE points", path, GD_MAXKDE);
      H.kt.push_back(lig_code(t[1]));
      for (int k = 0; k < 3; ++k) H.kxyz.push_back(to_f(t[2 + k]));
    } else if (tag == "PSP") {
      if (t.size() < 4) return fail(GD_E_INVALID, "%s: short PSP line", path);
      const int r = std::atoi(t[1].c_str()), l = lig_code(t[2]);
      if (r < 0 || r >= GD_MAXPRO) return fail(GD_E_CAPACITY, "%s: PSP residue %d outside [0, %d)", path, r, GD_MAXPRO);
      H.psp[(size_t)r * GD_MAXLIG + l] = to_f(t[3]);
    } else if (tag == "MCS") {
      if (H.nrow >= GD_MAX_MCS_ROW) return fail(GD_E_CAPACITY, "%s: more than %d MCS rows", path, GD_MAX_MCS_ROW);
      Mcs m;
      std::memset(&m, 0, sizeof(m));
      for (int j = 0; j < GD_MAX_MCS_COL; ++j) m.x[j] = m.y[j] = m.z[j] = GD_MCS_INVALID_COORD;
      std::vector<int> cols;
      std::vector<float> ent;
      if (t.size() > 1 && t[1] == id) {
        if (t.size() < 4) return fail(GD_E_INVALID, "%s: short MCS line", path);
        m.tcc = to_f(t[2]);
        m.ncol = std::atoi(t[3].c_str());
        if (m.ncol < 0 || t.size() < 4 + 4 * (size_t)m.ncol)
          return fail(GD_E_INVALID, "%s: MCS line with %d columns announced", path, m.ncol);
        for (int a = 0; a < m.ncol; ++a) {
          const int loc = std::atoi(t[4 * a + 4].c_str()) - 1;
          if (loc < 0 || loc >= GD_MAXLIG - 1) return fail(GD_E_INVALID, "%s: MCS position %d out of bounds", path, loc + 1);
          m.x[loc] = to_f(t[4 * a + 5]);
          m.y[loc] = to_f(t[4 * a + 6]);
          m.z[loc] = to_f(t[4 * a + 7]);
          cols.push_back(loc);
          ent.push_back(m.x[loc]);
          ent.push_back(m.y[loc]);
          ent.push_back(m.z[loc]);
        }
      }
      H.rows.push_back(m);
      H.cols.push_back(cols);
      H.entries.push_back(ent);
      ++H.nrow;  // every MCS line is a row, whichever ligand it names
    }
  }
  return GD_OK;
}

bool in_set(int v, std::initializer_list<int> set)
{
  for (int x : set)
    if (v == x) return true;
  return false;
}

struct ProteinIn {
  int npoint = 0, nres = 0, nconf = 0;
  std::vector<int> r, t, d, c;  // per point: residue index, point type, residue code, class
  std::vector<int> seq3;        // per residue: serial number
  std::vector<float> xyz;       // [nconf][npoint][3]
};

// loadPrtConf / loadProtein, load.C:482-1034
int read_pdb(const char *path, ProteinIn &P)
{
  std::vector<std::string> lines;
  GD_TRY(read_lines(path, lines));
  for (const auto &s : lines)
    if (field(s, 0, 6) == "ENDMDL") ++P.nconf;
  if (P.nconf < 1) return fail(GD_E_INVALID, "%s: no ENDMDL-terminated model", path);
  if (P.nconf > GD_MAX_CONF_PRT) return fail(GD_E_CAPACITY, "%s: %d models (limit %d)", path, P.nconf, GD_MAX_CONF_PRT);
  auto push = [&](int r, int t, int d, int c) {
    P.r.push_back(r);
    P.t.push_back(t);
    P.d.push_back(d);
    P.c.push_back(c);
  };
  // effective points of the first model: CA, peptide plate, side chain
  for (const auto &s : lines) {
    if (s.size() > 53) {
      if (field(s, 0, 6) != "ATOM  ") continue;
      if (field(s, 12, 4) != " CA ") continue;
      const int res = res_code(field(s, 17, 3));
      if (res < 0) return fail(GD_E_INVALID, "%s: unknown residue %s", path, field(s, 17, 3).c_str());
      P.seq3.push_back(std::atoi(field(s, 22, 4).c_str()));
      const int pnr = P.nres;
      push(pnr, 0, res, 0);
      if (pnr > 1) push(pnr - 1, 1, res, 1);
      int sc[2][2];
      const int ns = side_chain(res, sc);
      for (int k = 0; k < ns; ++k) push(pnr, sc[k][0], res, sc[k][1]);
      ++P.nres;
    } else if (field(s, 0, 6) == "ENDMDL") {
      break;
    }
  }
  P.npoint = (int)P.r.size();
  if (P.npoint > GD_MAXPRO) return fail(GD_E_CAPACITY, "%s: %d points (limit %d)", path, P.npoint, GD_MAXPRO);
  // coordinates: per model, the mean of the atoms each point stands for
  P.xyz.assign((size_t)P.nconf * P.npoint * 3, 0.f);
  auto in = [](const std::string &a, std::initializer_list<const char *> set) {
    for (const char *x : set)
      if (a == x) return true;
    return false;
  };
  for (int p = 0; p < P.npoint; ++p) {
    const int res_i = P.r[p], pt = P.t[p];
    const int serial = P.seq3[res_i];
    const int prev = res_i > 0 ? P.seq3[res_i - 1] : 0;
    const bool plate = pt == 1 && res_i > 0 && res_i < P.nres - 1;
    // The reference looks the previous residue up in the conformation record
    // of the model before the current one (load.C:851-852 with myprt moved at
    // each ENDMDL, :873); from the third model on that record is not filled
    // yet and the lookup yields serial 0, so a plate point of models >= 2
    // averages the N atom (and C/O atoms of a residue numbered 0, if any).
    // Kept so that the Complex is the one the reference builds.
    float sx = 0.f, sy = 0.f, sz = 0.f, sn = 0.f;
    int conf = 0;
    for (const auto &s : lines) {
      if (s.size() > 53) {
        if (field(s, 0, 6) != "ATOM  ") continue;
        const int ser = std::atoi(field(s, 22, 4).c_str());
        const std::string a = field(s, 12, 4);
        const float x = to_f(field(s, 30, 8)), y = to_f(field(s, 38, 8)), z = to_f(field(s, 46, 8));
        bool use = false;
        if (ser == serial) {
          if (pt == 0) use = a == " CA ";
          else if (in_set(pt, {2, 3, 4, 11, 14, 17, 18, 23, 24, 25})) use = !in(a, {" N  ", " CA ", " C  ", " O  "});
          else if (in_set(pt, {5, 7, 9, 12, 15, 19, 21, 26, 28}))
            use = !in(a, {" N  ", " CA ", " C  ", " O  ", " CB ", " CG "});
          else if (in_set(pt, {6, 8, 10, 13, 16, 20, 22, 27, 29})) use = in(a, {" CB ", " CG "});
        }
        const int prev_here = conf <= 1 ? prev : 0;
        if (plate && ((ser == serial && a == " N  ") || (ser == prev_here && (a == " C  " || a == " O  "))))
          use = true;
        if (use) {
          sx += x;
          sy += y;
          sz += z;
          sn += 1.0f;
        }
      } else if (field(s, 0, 6) == "ENDMDL") {
        if (sn > 0.f) {
          float *o = &P.xyz[((size_t)conf * P.npoint + p) * 3];
          o[0] = sx / sn;
          o[1] = sy / sn;
          o[2] = sz / sn;
        }
        sx = sy = sz = sn = 0.f;
        ++conf;
      }
    }
  }
  return GD_OK;
}

}  // namespace

extern "C" int gd_load_complex(const gd_load_args_t *a, Complex *cx)
{
  if (!a || !cx || !a->enepara0 || !a->enepara) return fail(GD_E_INVALID, "null argument");
  if (a->num_temp < 1 || a->num_temp > GD_MAX_TMP) return fail(GD_E_INVALID, "num_temp = %d", a->num_temp);
  if (!(a->floor_temp > 0.f) || !(a->ceiling_temp > 0.f)) return fail(GD_E_INVALID, "temperatures must be > 0");
  LigandIn L;
  LhmIn H;
  ProteinIn P;
  GD_TRY(read_sdf(a->lig_sdf, a->molid, L));
  GD_TRY(read_ff(a->lhm_ff, a->ligand_id, H));
  GD_TRY(read_pdb(a->prt_pdb, P));
  const long long nrep = (long long)L.nconf * P.nconf * a->num_temp;
  if (nrep > GD_MAX_REP) return fail(GD_E_CAPACITY, "%lld replicas (limit %d)", nrep, GD_MAX_REP);
  std::memset(cx, 0, sizeof(Complex));
  const EnePara0 &e0 = *a->enepara0;

  // KDE points sorted by type (OptimizeKde, util_optimize_soa.C:327-365)
  const int K = (int)H.kt.size();
  {
    std::vector<double> v(K);
    for (int k = 0; k < K; ++k) v[k] = H.kt[k];
    const std::vector<int> o = order_by(v);
    for (int k = 0; k < K; ++k) {
      cx->kde.t[k] = H.kt[o[k]];
      cx->kde.x[k] = H.kxyz[3 * o[k]];
      cx->kde.y[k] = H.kxyz[3 * o[k] + 1];
      cx->kde.z[k] = H.kxyz[3 * o[k] + 2];
    }
    cx->kde.kde_npoint = K;
  }

  // ligand conformations (OptimizeLigand, util_optimize_soa.C:37-177; the GPU
  // frontend keeps copy 1 in input order)
  {
    std::vector<double> tv(L.natom);
    for (int i = 0; i < L.natom; ++i) tv[i] = L.type[i];
    const std::vector<int> by_type = order_by(tv);
    for (int j = 0; j < L.nconf; ++j) {
      Ligand &g = cx->lig[j];
      const float *x = &L.xyz[(size_t)j * L.natom * 3];
      for (int k = 0; k < 3; ++k) g.center[k] = L.center[k];
      g.lig_natom = L.natom;
      for (int i = 0; i < L.natom; ++i) {
        g.x1[i] = g.x2[i] = x[3 * i];
        g.y1[i] = g.y2[i] = x[3 * i + 1];
        g.z1[i] = g.z2[i] = x[3 * i + 2];
        g.t1[i] = g.t2[i] = L.type[i];
        g.c1[i] = g.c2[i] = L.charge[i];
        const int s = by_type[i];
        g.x3[i] = x[3 * s];
        g.y3[i] = x[3 * s + 1];
        g.z3[i] = x[3 * s + 2];
        g.t3[i] = L.type[s];
        g.c3[i] = L.charge[s];
      }
      // KDE range per atom: first index of the type and the index where the run ends
      for (int i = 0; i < L.natom; ++i) {
        int st = 0, b = 0, e = 0;
        for (int k = 0; k < K; ++k) {
          const bool m = g.t3[i] == cx->kde.t[k];
          if (m && st == 0) st = 1, b = k;
          if (!m && st == 1) st = 2, e = k;
        }
        g.kde_begin_idx[i] = b;
        g.kde_end_idx[i] = e;
      }
    }
  }

  // protein conformations (OptimizeProtein, util_optimize_soa.C:181-270; SetPocketCenter, util.C:313-321)
  {
    std::vector<double> cv(P.npoint);
    for (int i = 0; i < P.npoint; ++i) cv[i] = P.c[i];
    const std::vector<int> by_class = order_by(cv);
    for (int j = 0; j < P.nconf; ++j) {
      Protein &q = cx->prt[j];
      q.prt_npoint = P.npoint;
      for (int k = 0; k < 3; ++k) q.pocket_center[k] = L.center[k];
      for (int i = 0; i < P.npoint; ++i) {
        const int s = by_class[i];
        const float *x = &P.xyz[((size_t)j * P.npoint + s) * 3];
        q.x[i] = x[0];
        q.y[i] = x[1];
        q.z[i] = x[2];
        q.t[i] = P.t[s];
        q.c[i] = P.c[s];
        q.ele[i] = e0.ele[P.t[s] == 0 ? P.d[s] + 30 : P.t[s]];
        q.seq3r[i] = P.seq3[P.r[s]];
        q.cdc[i] = (P.c[s] == 0 && P.d[s] == 12) || P.c[s] == 2;
        q.hpp[i] = e0.hpp[P.d[s]];
      }
    }
  }

  // pocket-specific potential, transposed (OptimizePsp, util_optimize_soa.C:278-285)
  for (int r = 0; r < GD_MAXPRO; ++r)
    for (int l = 0; l < GD_MAXLIG; ++l) cx->psp.psp[l][r] = H.psp[(size_t)r * GD_MAXLIG + l];

  // MCS rows and their sparse copies (OptimizeMcs, util_optimize_soa.C:371-460)
  {
    int ptr = 0;
    for (int i = 0; i < H.nrow; ++i) {
      cx->mcs[i] = H.rows[i];
      const int nc = H.rows[i].ncol;
      for (int k = 0; k < nc; ++k) {
        cx->mcs_ell.i[i][k] = H.cols[i][k];
        cx->mcs_ell.x[i][k] = H.entries[i][3 * k];
        cx->mcs_ell.y[i][k] = H.entries[i][3 * k + 1];
        cx->mcs_ell.z[i][k] = H.entries[i][3 * k + 2];
        cx->mcs_csr.idx_col[ptr + k] = H.cols[i][k];
        cx->mcs_csr.idx_row[ptr + k] = i;
        cx->mcs_csr.x[ptr + k] = H.entries[i][3 * k];
        cx->mcs_csr.y[ptr + k] = H.entries[i][3 * k + 1];
        cx->mcs_csr.z[ptr + k] = H.entries[i][3 * k + 2];
      }
      cx->mcs_ell.ncol[i] = nc;
      cx->mcs_ell.tcc[i] = H.rows[i].tcc;
      cx->mcs_csr.tcc[i] = H.rows[i].tcc;
      ptr += nc;
    }
    cx->mcs_csr.npoint = ptr;
  }

  // the parameter tables; the struct's tail padding stays zero
  std::memcpy(&cx->enepara, a->enepara, offsetof(EnePara, w) + sizeof(a->enepara->w));

  // temperature ladder (SetTemperature, util.C:326-355; k_B = 1; the ratio in
  // float arithmetic, as the reference's unqualified exp/log of floats)
  {
    const int n = a->num_temp;
    if (n == 1) {
      cx->temp[0].order = 0;
      cx->temp[0].minus_beta = 0.0f - 1.0f / (1.0f * a->floor_temp);
    } else {
      const float ratio = std::exp(std::log(a->ceiling_temp / a->floor_temp) / (float)(n - 1));
      float t = a->floor_temp;
      for (int i = 0; i < n; ++i) {
        cx->temp[i].order = i;
        cx->temp[i].minus_beta = 0.0f - 1.0f / (1.0f * t);
        t *= ratio;
      }
    }
  }

  ComplexSize &sz = cx->size;
  sz.n_lig = L.nconf;
  sz.n_prt = P.nconf;
  sz.n_tmp = a->num_temp;
  sz.n_rep = (int)nrep;
  sz.lig_natom = L.natom;
  sz.prt_npoint = P.npoint;
  sz.kde_npoint = K;
  sz.mcs_nrow = H.nrow;
  std::vector<ReplicaMC> reps;
  default_replicas(sz.n_lig, sz.n_prt, sz.n_tmp, reps);  // SetReplica, util.C:360-396
  for (int r = 0; r < sz.n_rep; ++r) cx->replica[r] = reps[r];

  McPara &mp = cx->mcpara;
  mp.steps_total = a->steps_total;
  mp.steps_per_dump = a->steps_per_dump;
  mp.steps_per_exchange = a->steps_per_exchange;
  for (int i = 0; i < 3; ++i) mp.move_scale[i] = a->translation_step;
  for (int i = 3; i < 6; ++i) mp.move_scale[i] = a->rotation_step;
  cx->rep_begin = 0;
  cx->rep_end = sz.n_rep - 1;
  return sz.n_rep;
}
