// Host-side domain initialisation: a C++ restatement of FDMAP's init_domain
// (domain.f90:45-378) and the time-loop set-up of main.f90:57-116, driven by
// FDMAP's own namelist input files.  It produces the fdmap_desc that a Fortran
// driver would hand to the GPU engine.  Only the features the time-stepping
// hot path supports are accepted; anything else is rejected with an error
// instead of being silently ignored.
#include "fdmap_host.h"

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "body_formulas.h"
#include "sbp_tables.h"

namespace {

thread_local std::string g_last_error;

struct InitError {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw InitError{code, msg}; }

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// ---------------------------------------------------------------------------
// Fortran namelist subset reader.
//
// Fortran's `read(unit, nml=name)` scans forward from the current record to
// the first group that starts with `&name` and reads `key = value` items up to
// the terminating '/'.  FDMAP positions the unit first (rewind, or
// seek_to_string, io.f90:209-228, which leaves it after the first line whose
// leading token equals the marker).  Both behaviours are reproduced here.
// ---------------------------------------------------------------------------
struct Namelist {
  bool found = false;
  std::map<std::string, std::vector<std::string>> kv;
};

// Position just past the line whose first token equals `marker`, or npos.
size_t seek_marker(const std::string& text, const std::string& marker) {
  size_t pos = 0;
  while (pos < text.size()) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    size_t a = pos;
    while (a < eol && (text[a] == ' ' || text[a] == '\t' || text[a] == '\r')) ++a;
    size_t b = a;
    while (b < eol && !std::isspace((unsigned char)text[b]) && text[b] != ',') ++b;
    if (text.compare(a, b - a, marker) == 0 && b - a == marker.size()) return eol;
    pos = eol + 1;
  }
  return std::string::npos;
}

// Tokens of a namelist group body.
struct Tok {
  enum Kind { IDENT, EQ, VAL, END } kind;
  std::string s;
};

Namelist read_nml(const std::string& text, size_t start, const std::string& name) {
  Namelist nl;
  if (start == std::string::npos) return nl;
  // locate "&name" (case-insensitive) at a token boundary, outside comments
  std::string key = "&" + lower(name);
  size_t pos = start;
  size_t gstart = std::string::npos;
  while (pos < text.size()) {
    size_t eol = text.find('\n', pos);
    if (eol == std::string::npos) eol = text.size();
    std::string line = lower(text.substr(pos, eol - pos));
    size_t a = line.find_first_not_of(" \t\r");
    if (a != std::string::npos && line.compare(a, key.size(), key) == 0) {
      size_t after = a + key.size();
      if (after >= line.size() || (!std::isalnum((unsigned char)line[after]) && line[after] != '_')) {
        gstart = pos + after;
        break;
      }
    }
    pos = eol + 1;
  }
  if (gstart == std::string::npos) return nl;
  nl.found = true;
  // tokenize until a '/' outside quotes
  std::vector<Tok> toks;
  size_t i = gstart;
  const size_t n = text.size();
  while (i < n) {
    char c = text[i];
    if (std::isspace((unsigned char)c) || c == ',') { ++i; continue; }
    if (c == '!') {  // comment to end of line
      while (i < n && text[i] != '\n') ++i;
      continue;
    }
    if (c == '/') break;
    if (c == '=') { toks.push_back({Tok::EQ, "="}); ++i; continue; }
    if (c == '\'' || c == '"') {
      char q = c;
      std::string s;
      ++i;
      while (i < n) {
        if (text[i] == q) {
          if (i + 1 < n && text[i + 1] == q) { s += q; i += 2; continue; }
          ++i;
          break;
        }
        s += text[i++];
      }
      toks.push_back({Tok::VAL, s});
      continue;
    }
    // bare word: identifier, number, logical, or repeat-count
    std::string s;
    while (i < n && !std::isspace((unsigned char)text[i]) && text[i] != ',' && text[i] != '=' &&
           text[i] != '/' && text[i] != '!')
      s += text[i++];
    // identifier followed by '=' is a key
    size_t j = i;
    while (j < n && (text[j] == ' ' || text[j] == '\t' || text[j] == '\r' || text[j] == '\n')) ++j;
    bool is_key = (j < n && text[j] == '=') &&
                  (std::isalpha((unsigned char)s[0]) || s[0] == '_');
    toks.push_back({is_key ? Tok::IDENT : Tok::VAL, s});
  }
  std::string cur;
  for (size_t k = 0; k < toks.size(); ++k) {
    if (toks[k].kind == Tok::IDENT) {
      cur = lower(toks[k].s);
      nl.kv[cur].clear();
      continue;
    }
    if (toks[k].kind == Tok::EQ) continue;
    if (cur.empty()) fail(FDMAP_ERR_INVALID_ARG, "namelist &" + name + ": value before any key");
    // r*c repeat counts
    const std::string& v = toks[k].s;
    size_t star = v.find('*');
    if (star != std::string::npos && star > 0 &&
        std::all_of(v.begin(), v.begin() + star, [](char ch) { return std::isdigit((unsigned char)ch); })) {
      int r = std::atoi(v.substr(0, star).c_str());
      for (int t = 0; t < r; ++t) nl.kv[cur].push_back(v.substr(star + 1));
    } else {
      nl.kv[cur].push_back(v);
    }
  }
  return nl;
}

double parse_real(const std::string& s0, const std::string& what) {
  std::string s = s0;
  for (auto& c : s)
    if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0') fail(FDMAP_ERR_INVALID_ARG, "bad real for " + what + ": '" + s0 + "'");
  return v;
}

bool parse_logical(const std::string& s0, const std::string& what) {
  std::string s = lower(s0);
  if (!s.empty() && s[0] == '.') s = s.substr(1);
  if (!s.empty() && (s[0] == 't')) return true;
  if (!s.empty() && (s[0] == 'f')) return false;
  fail(FDMAP_ERR_INVALID_ARG, "bad logical for " + what + ": '" + s0 + "'");
}

// Component lists of the derived types FDMAP reads positionally.
const std::map<std::string, std::vector<std::string>>& type_components() {
  static const std::map<std::string, std::vector<std::string>> t = {
      {"point", {"x", "y"}},
      {"fields_perturb", {"shape", "x0", "y0", "lx", "ly", "vx", "vy", "vz", "sxx", "sxy", "sxz", "syy", "syz", "szz"}},
      {"ratestate_constant", {"a", "b", "v0", "f0", "l", "fw", "vw"}},
      {"slipweak_constant", {"c0", "fs", "fd", "dc"}},
      {"kinematic", {"c0", "fd", "dfdx", "vl", "vr", "xl", "xr", "tmax"}},
      {"load", {"shape", "s", "n", "t", "r", "x0", "y0"}},
  };
  return t;
}

// Value lookup with `var%comp` and positional `var = v1, v2, ...` forms.
const std::string* nml_value(const Namelist& nl, const std::string& var, const std::string& type = "",
                             const std::string& comp = "") {
  std::string k = lower(var);
  if (!comp.empty()) {
    auto it = nl.kv.find(k + "%" + lower(comp));
    if (it != nl.kv.end() && !it->second.empty()) return &it->second[0];
    auto it2 = nl.kv.find(k);
    if (it2 != nl.kv.end()) {
      const auto& comps = type_components().at(type);
      for (size_t c = 0; c < comps.size(); ++c)
        if (comps[c] == lower(comp)) {
          if (c < it2->second.size()) return &it2->second[c];
          return nullptr;
        }
    }
    return nullptr;
  }
  auto it = nl.kv.find(k);
  if (it != nl.kv.end() && !it->second.empty()) return &it->second[0];
  return nullptr;
}

double get_real(const Namelist& nl, const std::string& var, double def, const std::string& type = "",
                const std::string& comp = "") {
  const std::string* v = nml_value(nl, var, type, comp);
  return v ? parse_real(*v, var + (comp.empty() ? "" : "%" + comp)) : def;
}
int get_int(const Namelist& nl, const std::string& var, int def) {
  const std::string* v = nml_value(nl, var);
  return v ? (int)std::lround(parse_real(*v, var)) : def;
}
bool get_bool(const Namelist& nl, const std::string& var, bool def) {
  const std::string* v = nml_value(nl, var);
  return v ? parse_logical(*v, var) : def;
}
std::string get_str(const Namelist& nl, const std::string& var, const std::string& def,
                    const std::string& type = "", const std::string& comp = "") {
  const std::string* v = nml_value(nl, var, type, comp);
  return v ? *v : def;
}
std::vector<int> get_int_list(const Namelist& nl, const std::string& var) {
  std::vector<int> out;
  auto it = nl.kv.find(lower(var));
  if (it != nl.kv.end())
    for (auto& s : it->second) out.push_back((int)std::lround(parse_real(s, var)));
  return out;
}

std::vector<double> read_binary_doubles(const std::string& path, size_t count, size_t offset_doubles = 0) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) fail(FDMAP_ERR_IO, "cannot open file " + path);
  std::vector<double> v(count);
  if (std::fseek(f, (long)(offset_doubles * sizeof(double)), SEEK_SET) != 0 ||
      std::fread(v.data(), sizeof(double), count, f) != count) {
    std::fclose(f);
    fail(FDMAP_ERR_IO, "short read from " + path);
  }
  std::fclose(f);
  return v;
}

// ---------------------------------------------------------------------------
// search_binary (utilities.f90:13-157, floor mode without initial guess); the
// shape functions of utilities.f90:303-420 are in body_formulas.h.
// ---------------------------------------------------------------------------
int search_floor(const double* x, int n, double y, bool* out) {
  // returns a 1-based index i with x(i) <= y < x(i+1)
  if (n == 1) {
    *out = !(y == x[0]);
    return 1;
  }
  int low = 1, high = n;
  if (y < x[low - 1]) { *out = true; return low; }
  if (y >= x[high - 1]) { *out = true; return high - 1; }
  *out = false;
  while (high - low > 1) {
    int mid = (low + high) / 2;
    if (x[mid - 1] <= y) low = mid; else high = mid;
  }
  return low;
}

// ---------------------------------------------------------------------------
// The domain object
// ---------------------------------------------------------------------------
struct Curve {
  std::vector<double> x, y, n1, n2;  // indexed 0..n-1 along the side
};

struct SideStore {
  std::vector<double> M, F0, normal, x, y;
};

struct BlockIn {
  int nx = 1, ny = 1, mgx = 1, mgy = 1, iblock_x = 0, iblock_y = 0, pgx = 1, pgy = 1;
  double LB[2], LT[2], RB[2], RT[2];
  std::string bndfile[4];
  double bndmap[4] = {0, 0, 0, 0};
  int bc[4] = {FDMAP_BC_NONE, FDMAP_BC_NONE, FDMAP_BC_NONE, FDMAP_BC_NONE};
  // material (material.f90:29-149)
  bool heterogeneous = false;
  std::string medium_file;
  double rho = 0, G = 0, cs = 0, cp = 0, M = 0, gamma = 0, nu = 0, Zs = 0, Zp = 0;
  double F0v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double Cdiss = 0;  // operator_list (domain.f90:172-180), scaled by CFL/dt after set_dt
  // pml_list (init_pml, material.f90:152-222)
  bool pmlx = false, pmly = false;
  double pml_n = 0, pml_sigma = 0, pml_kappa = 0, pml_mx = 0, pml_px = 0, pml_my = 0, pml_py = 0;
  Curve curve[4];
  SideStore side[4];
  std::vector<double> side_mat[4];  // on-device body of a heterogeneous block: rho, cs, cp at side nodes
};

struct FrictionStore {
  std::vector<double> a, b, V0, f0, L, fw, Vw, c0, fs, fd, Dc, bsS0, bsN0;
  std::vector<double> V, O, S, N, S0, N0, Ds, Dn, DDs, DDn, Psi, DPsi, D, trup, W, DW, Nreg, DNreg;
};

struct IfaceStore {
  std::vector<double> nhat, x, y;
  FrictionStore fr;
};

}  // namespace

struct fdmap_domain {
  fdmap_desc desc{};
  std::vector<fdmap_block> blocks;
  std::vector<fdmap_iface> ifaces;
  std::vector<BlockIn> bin;
  std::vector<IfaceStore> istore;
  std::vector<double> F, DF, x, y, xq, xr, yq, yr, J, Ji;
  std::vector<double> rho, cs, cp, G, M, gamma, nu;
  // on-device initialisation: the recipe the engine builds the body from
  bool dev_body = false;
  fdmap_body body{};
  std::string forcing_path;  // source_list forcing_filename, resolved
  std::vector<fdmap_block_body> bbody;
};

namespace {

inline size_t gidx(const fdmap_desc& d, int i, int j) { return (size_t)(i - 1) + (size_t)d.nx * (size_t)(j - 1); }

int bc_code(const std::string& bc) {
  std::string b = lower(bc);
  if (b == "none") return FDMAP_BC_NONE;
  if (b == "absorbing") return FDMAP_BC_ABSORBING;
  if (b == "free") return FDMAP_BC_FREE;
  if (b == "rigid") return FDMAP_BC_RIGID;
  if (b == "absorbing-0") return FDMAP_BC_ABSORBING_0;
  if (b == "free-0") return FDMAP_BC_FREE_0;
  if (b == "rigid-0") return FDMAP_BC_RIGID_0;
  if (b == "absorbing-velocity") return FDMAP_BC_ABSORBING_VELOCITY;
  if (b == "free-velocity") return FDMAP_BC_FREE_VELOCITY;
  fail(FDMAP_ERR_UNSUPPORTED, "boundary condition '" + bc + "' is not supported");
}

int law_code(const std::string& law) {
  if (law == "frictionless") return FDMAP_FR_FRICTIONLESS;
  if (law == "locked") return FDMAP_FR_LOCKED;
  if (law == "SW") return FDMAP_FR_SW;
  if (law == "SL") return FDMAP_FR_SL;
  if (law == "FL") return FDMAP_FR_FL;
  if (law == "RSL") return FDMAP_FR_RSL;
  if (law == "RFL") return FDMAP_FR_RFL;
  if (law == "RSF") return FDMAP_FR_RSF;
  if (law == "RAL") return FDMAP_FR_RAL;
  fail(FDMAP_ERR_UNSUPPORTED, "friction law '" + law + "' is not supported");
}

int ld_code(const std::string& s) {
  if (s == "") return FDMAP_LD_NONE;
  if (s == "uniform") return FDMAP_LD_UNIFORM;
  if (s == "linear") return FDMAP_LD_LINEAR;
  if (s == "boxcar") return FDMAP_LD_BOXCAR;
  if (s == "smooth_boxcar") return FDMAP_LD_SMOOTH_BOXCAR;
  if (s == "triangle") return FDMAP_LD_TRIANGLE;
  if (s == "smooth") return FDMAP_LD_SMOOTH;
  if (s == "gaussian") return FDMAP_LD_GAUSSIAN;
  fail(FDMAP_ERR_UNSUPPORTED, "load shape '" + s + "' is not supported");
}

int stf_code(const std::string& s) {
  if (s == "ramp") return FDMAP_STF_RAMP;
  if (s == "sinusoid") return FDMAP_STF_SINUSOID;
  if (s == "gaussian") return FDMAP_STF_GAUSSIAN;
  if (s == "Ricker") return FDMAP_STF_RICKER;
  fail(FDMAP_ERR_UNSUPPORTED, "source time function '" + s + "' is not supported");
}

std::string join_path(const std::string& base, const std::string& f) {
  if (f.empty() || f[0] == '/' || base.empty()) return f;
  return base + "/" + f;
}

// line_map (geometry.f90:70-106): nodes m..p of a straight (optionally
// stretched) edge from P1 to P2 over the index coordinate t in [t1, t2].
void line_map(Curve& C, const double P1[2], const double P2[2], int m, int p, double t1, double t2, double B) {
  int n = p - m + 1;
  C.x.assign(n, 0); C.y.assign(n, 0); C.n1.assign(n, 0); C.n2.assign(n, 0);
  for (int k = 0; k < n; ++k) {
    double t = (double)(m + k);
    double w = (t - t1) / (t2 - t1);
    if (B > 0.0) w = 1.0 + std::tanh(B * (w - 1.0)) / std::tanh(B);
    else if (B < 0.0) w = std::tanh(B * w) / std::tanh(B);
    C.x[k] = P1[0] + (P2[0] - P1[0]) * w;
    C.y[k] = P1[1] + (P2[1] - P1[1]) * w;
  }
  double L = std::sqrt((P2[0] - P1[0]) * (P2[0] - P1[0]) + (P2[1] - P1[1]) * (P2[1] - P1[1]));
  if (L != 0) {
    for (int k = 0; k < n; ++k) {
      C.n1[k] = (P2[1] - P1[1]) / L;
      C.n2[k] = (P1[0] - P2[0]) / L;
    }
  } else {
    std::fill(C.n1.begin(), C.n1.end(), 1e40);
    std::fill(C.n2.begin(), C.n2.end(), 1e40);
  }
}

// read_bnd (grid.f90:646-702): x, y, n1, n2 arrays of length n, real*8.
void read_curve(Curve& C, const std::string& path, int n) {
  std::vector<double> v = read_binary_doubles(path, (size_t)4 * n);
  C.x.assign(v.begin(), v.begin() + n);
  C.y.assign(v.begin() + n, v.begin() + 2 * n);
  C.n1.assign(v.begin() + 2 * n, v.begin() + 3 * n);
  C.n2.assign(v.begin() + 3 * n, v.begin() + 4 * n);
}

// SBP derivative with unit spacing (fd.f90:42-80) of f over the block range
// [mg, pg]; f and Df are indexed 0..n-1 (n = pg-mg+1).
void sbp_diff(const fdmap::SbpOperator& op, const std::vector<double>& f, std::vector<double>& Df) {
  int n = (int)f.size();
  Df.assign(n, 0.0);
  if (n == 1) return;
  for (int r = 0; r < op.nbst; ++r) {
    double s = 0.0;
    for (int k = 0; k < op.nbnd; ++k) s = s + op.DL[r][k] * f[k];
    Df[r] = s;
  }
  for (int r = 0; r < op.nbst; ++r) {
    // DR(:,-r) = -DL(nbnd-1:0:-1, r) applied to f(pg-nbnd+1:pg)
    double s = 0.0;
    for (int k = 0; k < op.nbnd; ++k) {
      double w = -op.DL[r][op.nbnd - 1 - k];
      s = s + w * f[n - op.nbnd + k];
    }
    Df[n - 1 - r] = s;
  }
  for (int i = op.nbst; i <= n - 1 - op.nbst; ++i) {
    // dot_product(DI(mI:pI), f(i+mI:i+pI)), summed from s = mI upward
    double s = 0.0;
    for (int q = -op.pI; q <= op.pI; ++q) {
      double w = q < 0 ? -op.DI[-q] : (q == 0 ? 0.0 : op.DI[q]);
      s = s + w * f[i + q];
    }
    Df[i] = s;
  }
}

// one coordinate (c = 0: x, 1: y) of node (i, j) of block B, interpolated
// from its four edge curves (transfinite_interp, geometry.f90:153-200)
double node_coord(const BlockIn& B, int i, int j, int c) {
  double qmin = B.mgx, qmax = B.pgx, rmin = B.mgy, rmax = B.pgy;
  double Wq = qmax - qmin, Wr = rmax - rmin;
  if (Wq == 0.0) Wq = 1.0;
  if (Wr == 0.0) Wr = 1.0;
  const std::vector<double>& cL = c ? B.curve[0].y : B.curve[0].x;
  const std::vector<double>& cR = c ? B.curve[1].y : B.curve[1].x;
  const std::vector<double>& cB = c ? B.curve[2].y : B.curve[2].x;
  const std::vector<double>& cT = c ? B.curve[3].y : B.curve[3].x;
  return fdmap::transfinite((double)i, (double)j, qmin, qmax, rmin, rmax, Wq, Wr, cL[j - B.mgy], cR[j - B.mgy],
                            cB[i - B.mgx], cT[i - B.mgx], B.LB[c], B.LT[c], B.RB[c], B.RT[c]);
}

struct Perturb {
  std::string shape;
  int code = FDMAP_PERTURB_NONE;
  double x0 = 0, y0 = 0, Lx = 1, Ly = 1;
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // vx vy vz sxx sxy sxz syy syz szz
};

Perturb read_perturb(const Namelist& nl, const std::string& name) {
  Perturb P;
  P.shape = get_str(nl, name, "", "fields_perturb", "shape");
  P.x0 = get_real(nl, name, 0, "fields_perturb", "x0");
  P.y0 = get_real(nl, name, 0, "fields_perturb", "y0");
  P.Lx = get_real(nl, name, 1, "fields_perturb", "lx");
  P.Ly = get_real(nl, name, 1, "fields_perturb", "ly");
  const char* comps[9] = {"vx", "vy", "vz", "sxx", "sxy", "sxz", "syy", "syz", "szz"};
  for (int c = 0; c < 9; ++c) P.v[c] = get_real(nl, name, 0, "fields_perturb", comps[c]);
  if (P.shape == "") P.code = FDMAP_PERTURB_NONE;
  else if (P.shape == "linear") P.code = FDMAP_PERTURB_LINEAR;
  else if (P.shape == "boxcar") P.code = FDMAP_PERTURB_BOXCAR;
  else if (P.shape == "triangle") P.code = FDMAP_PERTURB_TRIANGLE;
  else if (P.shape == "smooth") P.code = FDMAP_PERTURB_SMOOTH;
  else if (P.shape == "gaussian") P.code = FDMAP_PERTURB_GAUSSIAN;
  else fail(FDMAP_ERR_UNSUPPORTED, "perturbation shape '" + P.shape + "' is not supported");
  return P;
}

// perturb_fields (fields.f90:900-934)
double perturb_amp(double x, double y, const Perturb& P) {
  return fdmap::perturb_amp(P.code, x, y, P.x0, P.y0, P.Lx, P.Ly);
}

// field vector of a perturbation in the mode's field order
void perturb_vector(const Perturb& P, int mode, double* out) {
  if (mode == 2) {
    const int idx[6] = {0, 1, 3, 4, 6, 8};  // vx vy sxx sxy syy szz
    for (int l = 0; l < 6; ++l) out[l] = P.v[idx[l]];
  } else {
    const int idx[3] = {2, 5, 7};  // vz sxz syz
    for (int l = 0; l < 3; ++l) out[l] = P.v[idx[l]];
  }
}

void build(fdmap_domain& dom, const std::string& text, const std::string& base, bool dev_body) {
  fdmap_desc& d = dom.desc;

  // ---- problem_list (main.f90:57-78)
  Namelist pl = read_nml(text, 0, "problem_list");
  double t0 = get_real(pl, "t", 0.0);
  int nt = get_int(pl, "nt", 0);
  double CFL = get_real(pl, "cfl", 0.0);
  double dt = get_real(pl, "dt", 0.0);
  double refine = get_real(pl, "refine", 1.0);
  double tend = get_real(pl, "tend", 0.0);
  std::string rkmethod = get_str(pl, "rkmethod", "LS");
  int rkorder = get_int(pl, "rkorder", 3);
  if (rkmethod != "LS") fail(FDMAP_ERR_UNSUPPORTED, "RKmethod must be 'LS'");
  if (!get_bool(pl, "solid", true)) fail(FDMAP_ERR_UNSUPPORTED, "solid=F is not supported");
  fdmap::RkTable rk;
  if (!fdmap::rk_table(rkorder, &rk)) fail(FDMAP_ERR_INVALID_ARG, "Invalid Runge-Kutta order");

  // ---- domain_list (domain.f90:84-139)
  Namelist dl = read_nml(text, 0, "domain_list");
  int mode = get_int(dl, "mode", 2);
  std::string fdm = get_str(dl, "fdmethod", "SBP6");
  int nbx = get_int(dl, "nblocks_x", 0), nby = get_int(dl, "nblocks_y", 0), nblocks = get_int(dl, "nblocks", 0);
  if (get_bool(dl, "exact_metric", false)) fail(FDMAP_ERR_UNSUPPORTED, "exact_metric=T is not supported");
  if (get_bool(dl, "operator_split", false)) fail(FDMAP_ERR_UNSUPPORTED, "operator_split=T is not supported");
  if (get_bool(dl, "acoustic_gravity_waves", false) || get_bool(dl, "basal_traction_plane_stress", false))
    fail(FDMAP_ERR_UNSUPPORTED, "acoustic gravity / basal traction terms are not supported");
  d.energy_balance = get_bool(dl, "energy_balance", false) ? 1 : 0;
  d.displacement = get_bool(dl, "displacement", false) ? 1 : 0;
  d.peak = get_bool(dl, "peak", false) ? 1 : 0;
  std::vector<int> nx_list = get_int_list(dl, "nx_list"), ny_list = get_int_list(dl, "ny_list");
  if (mode != 2 && mode != 3) fail(FDMAP_ERR_INVALID_ARG, "mode must be 2 or 3");
  int method;
  if (fdm == "SBP2") method = FDMAP_SBP2;
  else if (fdm == "SBP4") method = FDMAP_SBP4;
  else if (fdm == "SBP6") method = FDMAP_SBP6;
  else fail(FDMAP_ERR_UNSUPPORTED, "FDmethod '" + fdm + "' is not supported");
  fdmap::SbpOperator op;
  fdmap::sbp_operator(method, &op);
  if (nbx == 0) nbx = 1;
  if (nby == 0) nby = 1;
  if (nblocks == 0) nblocks = nbx * nby;
  if (nblocks != nbx * nby) fail(FDMAP_ERR_UNSUPPORTED, "nblocks must equal nblocks_x*nblocks_y");
  int nifaces = (nbx - 1) * nby + (nby - 1) * nbx;
  d.mode = mode;
  d.nF = mode == 2 ? 6 : 3;
  d.fd_method = method;
  d.rk_order = rkorder;
  d.nblocks = nblocks;
  d.nifaces = nifaces;
  const int nF = d.nF;

  // ---- per-block lists
  dom.bin.resize(nblocks);
  for (int b = 0; b < nblocks; ++b) {
    BlockIn& B = dom.bin[b];
    size_t mk = seek_marker(text, "!---BLOCK" + std::to_string(b + 1) + "---");
    if (mk == std::string::npos) fail(FDMAP_ERR_INVALID_ARG, "String '!---BLOCK" + std::to_string(b + 1) + "---' not found in file");
    Namelist ol = read_nml(text, mk, "operator_list");
    B.Cdiss = get_real(ol, "cdiss", 0.0);
    // pml_list defaults: no layer, sigma = kappa = 0, bounds at -/+huge(0d0).
    // The reference gives n no default; n = 0 (constant sigma) here.
    Namelist pml = read_nml(text, mk, "pml_list");
    B.pmlx = get_bool(pml, "pmlx", false);
    B.pmly = get_bool(pml, "pmly", false);
    B.pml_n = get_real(pml, "n", 0.0);
    B.pml_sigma = get_real(pml, "sigma", 0.0);
    B.pml_kappa = get_real(pml, "kappa", 0.0);
    B.pml_mx = get_real(pml, "mx", -DBL_MAX);
    B.pml_px = get_real(pml, "px", DBL_MAX);
    B.pml_my = get_real(pml, "my", -DBL_MAX);
    B.pml_py = get_real(pml, "py", DBL_MAX);
    Namelist gl = read_nml(text, mk, "grid_list");
    B.nx = get_int(gl, "nx", 1);
    B.ny = get_int(gl, "ny", 1);
    const char* cn[4] = {"lb", "lt", "rb", "rt"};
    double* cp_[4] = {B.LB, B.LT, B.RB, B.RT};
    for (int c = 0; c < 4; ++c) {
      cp_[c][0] = get_real(gl, cn[c], HUGE_VAL, "point", "x");
      cp_[c][1] = get_real(gl, cn[c], HUGE_VAL, "point", "y");
    }
    const char* sn[4] = {"L", "R", "B", "T"};
    for (int s = 0; s < 4; ++s) {
      B.bndfile[s] = get_str(gl, std::string("bnd") + sn[s] + "file", "");
      B.bndmap[s] = get_real(gl, std::string("bnd") + sn[s] + "map", 0.0);
    }
    Namelist bl = read_nml(text, mk, "boundaries_list");
    for (int s = 0; s < 4; ++s) B.bc[s] = bc_code(get_str(bl, std::string("bc") + sn[s], "none"));
    Namelist ml = read_nml(text, mk, "material_list");
    std::string response = get_str(ml, "response", "elastic");
    if (response != "elastic") fail(FDMAP_ERR_UNSUPPORTED, "material response '" + response + "' is not supported");
    B.heterogeneous = get_bool(ml, "heterogeneous", false);
    B.medium_file = get_str(ml, "filename", "");
    B.rho = get_real(ml, "rho", 0.0);
    B.G = get_real(ml, "g", 0.0);
    B.cs = get_real(ml, "cs", 0.0);
    B.cp = get_real(ml, "cp", 0.0);
  }

  // nx_list/ny_list, set_grid_indices, set_refine, set_grid (domain.f90:1538-1644, grid.f90:110-148)
  if (!nx_list.empty() && !ny_list.empty() && nx_list[0] != 0 && ny_list[0] != 0) {
    if ((int)nx_list.size() < nbx || (int)ny_list.size() < nby) fail(FDMAP_ERR_INVALID_ARG, "incorrect number of elements in nx_list/ny_list");
    for (int ix = 0; ix < nbx; ++ix)
      for (int iy = 0; iy < nby; ++iy) {
        dom.bin[ix + iy * nbx].nx = nx_list[ix];
        dom.bin[ix + iy * nbx].ny = ny_list[iy];
      }
  }
  {
    std::vector<int> mgx(nbx), mgy(nby);
    mgx[0] = 1; mgy[0] = 1;
    for (int ix = 1; ix < nbx; ++ix) mgx[ix] = mgx[ix - 1] + dom.bin[ix - 1].nx;
    for (int iy = 1; iy < nby; ++iy) mgy[iy] = mgy[iy - 1] + dom.bin[(iy - 1) * nbx].ny;
    for (int ix = 0; ix < nbx; ++ix)
      for (int iy = 0; iy < nby; ++iy) {
        BlockIn& B = dom.bin[ix + iy * nbx];
        B.mgx = mgx[ix]; B.mgy = mgy[iy]; B.iblock_x = ix + 1; B.iblock_y = iy + 1;
      }
  }
  for (auto& B : dom.bin) {
    int nx = B.nx, ny = B.ny;
    if (nx != 1) nx = (int)std::ceil((double)(nx - 1) * refine) + 1;
    if (ny != 1) ny = (int)std::ceil((double)(ny - 1) * refine) + 1;
    B.mgx = (int)std::ceil((double)(B.mgx - B.iblock_x) * refine) + B.iblock_x;
    B.mgy = (int)std::ceil((double)(B.mgy - B.iblock_y) * refine) + B.iblock_y;
    B.nx = nx; B.ny = ny;
    B.pgx = B.mgx + nx - 1;
    B.pgy = B.mgy + ny - 1;
  }
  int NX = 0, NY = 0;
  for (int ix = 0; ix < nbx; ++ix) NX += dom.bin[ix].nx;
  for (int iy = 0; iy < nby; ++iy) NY += dom.bin[iy * nbx].ny;
  d.nx = NX; d.ny = NY;
  const size_t NN = (size_t)NX * NY;

  // ---- grids (init_grid + interp_block, grid.f90:188-462)
  int minpts = op.nbst == 1 ? 3 : (op.nbst == 4 ? 8 : 12);
  if (!dev_body) {
    dom.x.assign(NN, 1e40); dom.y.assign(NN, 1e40);
    dom.xq.assign(NN, 1.0); dom.xr.assign(NN, 0.0); dom.yq.assign(NN, 0.0); dom.yr.assign(NN, 1.0);
    dom.J.assign(NN, 1.0); dom.Ji.assign(NN, 1.0);
  }
  for (int b = 0; b < nblocks; ++b) {
    BlockIn& B = dom.bin[b];
    if (B.nx < minpts || B.ny < minpts)
      fail(FDMAP_ERR_UNSUPPORTED, "block " + std::to_string(b + 1) + " has too few points for " + fdm +
                                      " (one-dimensional blocks are not supported)");
    double qmin = B.mgx, qmax = B.pgx, rmin = B.mgy, rmax = B.pgy;
    // L, R edges along r; B, T edges along q
    if (B.bndfile[0].empty()) line_map(B.curve[0], B.LB, B.LT, B.mgy, B.pgy, rmin, rmax, B.bndmap[0]);
    else read_curve(B.curve[0], join_path(base, B.bndfile[0]), B.ny);
    for (int k = 0; k < B.ny; ++k) { B.curve[0].n1[k] = -B.curve[0].n1[k]; B.curve[0].n2[k] = -B.curve[0].n2[k]; }
    if (B.bndfile[1].empty()) line_map(B.curve[1], B.RB, B.RT, B.mgy, B.pgy, rmin, rmax, B.bndmap[1]);
    else read_curve(B.curve[1], join_path(base, B.bndfile[1]), B.ny);
    if (B.bndfile[2].empty()) line_map(B.curve[2], B.LB, B.RB, B.mgx, B.pgx, qmin, qmax, B.bndmap[2]);
    else read_curve(B.curve[2], join_path(base, B.bndfile[2]), B.nx);
    if (B.bndfile[3].empty()) line_map(B.curve[3], B.LT, B.RT, B.mgx, B.pgx, qmin, qmax, B.bndmap[3]);
    else read_curve(B.curve[3], join_path(base, B.bndfile[3]), B.nx);
    for (int k = 0; k < B.nx; ++k) { B.curve[3].n1[k] = -B.curve[3].n1[k]; B.curve[3].n2[k] = -B.curve[3].n2[k]; }
    // transfinite_interp (geometry.f90:153-200); left to the device when it builds the body
    if (dev_body) continue;
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        dom.x[gidx(d, i, j)] = node_coord(B, i, j, 0);
        dom.y[gidx(d, i, j)] = node_coord(B, i, j, 1);
      }
  }

  // ---- metrics (init_grid_partials, grid.f90:465-618)
  double hmin = 1e40, hmax = 0.0;
  for (int b = 0; b < nblocks && !dev_body; ++b) {
    BlockIn& B = dom.bin[b];
    std::vector<double> f, Df;
    for (int j = B.mgy; j <= B.pgy; ++j) {
      f.resize(B.nx);
      for (int i = B.mgx; i <= B.pgx; ++i) f[i - B.mgx] = dom.x[gidx(d, i, j)];
      sbp_diff(op, f, Df);
      for (int i = B.mgx; i <= B.pgx; ++i) dom.xq[gidx(d, i, j)] = Df[i - B.mgx];
      for (int i = B.mgx; i <= B.pgx; ++i) f[i - B.mgx] = dom.y[gidx(d, i, j)];
      sbp_diff(op, f, Df);
      for (int i = B.mgx; i <= B.pgx; ++i) dom.yq[gidx(d, i, j)] = Df[i - B.mgx];
    }
    for (int i = B.mgx; i <= B.pgx; ++i) {
      f.resize(B.ny);
      for (int j = B.mgy; j <= B.pgy; ++j) f[j - B.mgy] = dom.x[gidx(d, i, j)];
      sbp_diff(op, f, Df);
      for (int j = B.mgy; j <= B.pgy; ++j) dom.xr[gidx(d, i, j)] = Df[j - B.mgy];
      for (int j = B.mgy; j <= B.pgy; ++j) f[j - B.mgy] = dom.y[gidx(d, i, j)];
      sbp_diff(op, f, Df);
      for (int j = B.mgy; j <= B.pgy; ++j) dom.yr[gidx(d, i, j)] = Df[j - B.mgy];
    }
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = gidx(d, i, j);
        dom.J[g] = dom.xq[g] * dom.yr[g] - dom.xr[g] * dom.yq[g];
        dom.Ji[g] = 1.0 / dom.J[g];
      }
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = gidx(d, i, j);
        double dxv = fdmap::spacing_q(dom.J[g], dom.xr[g], dom.yr[g]);
        double dyv = fdmap::spacing_r(dom.J[g], dom.xq[g], dom.yq[g]);
        hmin = std::min(hmin, std::min(dxv, dyv));
        hmax = std::max(hmax, std::max(dxv, dyv));
      }
  }

  // ---- material (init_material / init_medium, material.f90:29-149, 226-275)
  bool any_het = false;
  std::string medium_file;
  for (auto& B : dom.bin)
    if (B.heterogeneous && !any_het) { any_het = true; medium_file = B.medium_file; }
  if (any_het) {
    std::vector<double> v = read_binary_doubles(join_path(base, medium_file), 3 * NN);
    dom.rho.assign(v.begin(), v.begin() + NN);
    dom.cs.assign(v.begin() + NN, v.begin() + 2 * NN);
    dom.cp.assign(v.begin() + 2 * NN, v.begin() + 3 * NN);
    dom.G.resize(NN); dom.M.resize(NN); dom.gamma.resize(NN); dom.nu.resize(NN);
    for (size_t g = 0; g < NN; ++g) {
      dom.G[g] = dom.rho[g] * (dom.cs[g] * dom.cs[g]);
      dom.M[g] = dom.rho[g] * (dom.cp[g] * dom.cp[g]);
      dom.gamma[g] = 1.0 - 2.0 * ((dom.cs[g] / dom.cp[g]) * (dom.cs[g] / dom.cp[g]));
      dom.nu[g] = 0.5 * (dom.M[g] - 2.0 * dom.G[g]) / (dom.M[g] - dom.G[g]);
    }
  }
  // energy_block weights every block, heterogeneous ones too, with the
  // block's material_list constants (M%rho, M%G, M%lambda; energy.f90:67-90)
  for (auto& B : dom.bin) {
    if (B.cs == 0.0 && !B.heterogeneous) fail(FDMAP_ERR_INVALID_ARG, "Must specify S-wave speed");
    if (B.cp == 0.0) B.cp = std::sqrt(3.0) * B.cs;
    if (B.rho == 0.0) B.rho = B.G / (B.cs * B.cs);
    if (B.G == 0.0) B.G = B.rho * (B.cs * B.cs);
    B.M = B.rho * (B.cp * B.cp);
    double lambda = B.M - 2.0 * B.G;
    B.nu = 0.5 * lambda / (lambda + B.G);
    B.gamma = 1.0 - 2.0 * ((B.cs / B.cp) * (B.cs / B.cp));
    B.Zs = B.rho * B.cs;
    B.Zp = B.rho * B.cp;
  }

  // ---- fields (init_fields, fields.f90:57-278, 774-897)
  if (!dev_body) {
    dom.F.assign(NN * nF, 1e40);
    dom.DF.assign(NN * nF, 1e40);
  } else {
    dom.bbody.assign(nblocks, fdmap_block_body{});
  }
  for (int b = 0; b < nblocks; ++b) {
    BlockIn& B = dom.bin[b];
    size_t mk = seek_marker(text, "!---BLOCK" + std::to_string(b + 1) + "---");
    Namelist fl = read_nml(text, mk, "fields_list");
    std::string problem = get_str(fl, "problem", "");
    double vx0 = get_real(fl, "vx0", 0), vy0 = get_real(fl, "vy0", 0), vz0 = get_real(fl, "vz0", 0);
    double sxx0 = get_real(fl, "sxx0", 0), sxy0 = get_real(fl, "sxy0", 0), sxz0 = get_real(fl, "sxz0", 0);
    double syy0 = get_real(fl, "syy0", 0), syz0 = get_real(fl, "syz0", 0), szz0 = get_real(fl, "szz0", 0);
    double Psi = get_real(fl, "psi", 0);
    if (get_bool(fl, "prestress_from_file", false) || get_bool(fl, "initial_condition_from_file", false))
      fail(FDMAP_ERR_UNSUPPORTED, "prestress/initial condition from file is not supported");
    if (problem == "uniform") {
      if (Psi == 45.0) sxx0 = syy0;
      else sxx0 = (1.0 - 2.0 * sxy0 / (syy0 * std::tan(2.0 * (Psi * 0.017453292519943)))) * syy0;
      szz0 = 0.5 * (sxx0 + syy0);
    } else if (problem != "") {
      fail(FDMAP_ERR_UNSUPPORTED, "fields problem '" + problem + "' is not supported");
    }
    const double f0v[9] = {vx0, vy0, vz0, sxx0, sxy0, sxz0, syy0, syz0, szz0};
    for (int q = 0; q < 9; ++q) B.F0v[q] = f0v[q];
    Perturb P[5];
    for (int k = 0; k < 5; ++k) P[k] = read_perturb(fl, "p" + std::to_string(k + 1));
    double F0[6], Pv[5][6];
    if (mode == 2) { F0[0] = vx0; F0[1] = vy0; F0[2] = sxx0; F0[3] = sxy0; F0[4] = syy0; F0[5] = szz0; }
    else { F0[0] = vz0; F0[1] = sxz0; F0[2] = syz0; }
    for (int k = 0; k < 5; ++k) perturb_vector(P[k], mode, Pv[k]);
    if (dev_body) {
      fdmap_block_body& bb = dom.bbody[b];
      for (int l = 0; l < nF; ++l) bb.F0[l] = F0[l];
      for (int k = 0; k < 5; ++k) {
        bb.p[k].shape = P[k].code;
        bb.p[k].x0 = P[k].x0; bb.p[k].y0 = P[k].y0; bb.p[k].Lx = P[k].Lx; bb.p[k].Ly = P[k].Ly;
        for (int l = 0; l < nF; ++l) bb.p[k].v[l] = Pv[k][l];
      }
    }
    // sides (P1..P4 only)
    for (int s = 0; s < 4; ++s) {
      const Curve& c = B.curve[s];
      int n = (s < 2) ? B.ny : B.nx;
      SideStore& S = B.side[s];
      S.F0.assign((size_t)n * nF, 1e40);
      for (int k = 0; k < n; ++k) {
        double A[4];
        for (int q = 0; q < 4; ++q) A[q] = perturb_amp(c.x[k], c.y[k], P[q]);
        for (int l = 0; l < nF; ++l)
          S.F0[k + (size_t)n * l] = F0[l] + A[0] * Pv[0][l] + A[1] * Pv[1][l] + A[2] * Pv[2][l] + A[3] * Pv[3][l];
      }
    }
    // interior (P1..P5); left to the device when it builds the body
    if (dev_body) continue;
    for (int j = B.mgy; j <= B.pgy; ++j)
      for (int i = B.mgx; i <= B.pgx; ++i) {
        size_t g = gidx(d, i, j);
        double A[5];
        for (int q = 0; q < 5; ++q) A[q] = perturb_amp(dom.x[g], dom.y[g], P[q]);
        for (int l = 0; l < nF; ++l)
          dom.F[g + NN * l] = F0[l] + A[0] * Pv[0][l] + A[1] * Pv[1][l] + A[2] * Pv[2][l] + A[3] * Pv[3][l] + A[4] * Pv[4][l];
      }
  }

  // ---- edges (init_edges, domain.f90:1349-1459)
  for (auto& B : dom.bin) {
    for (int s = 0; s < 4; ++s) {
      int n = (s < 2) ? B.ny : B.nx;
      SideStore& S = B.side[s];
      S.normal.resize((size_t)n * 2);
      S.x = B.curve[s].x;
      S.y = B.curve[s].y;
      if (dev_body) {
        // the device derives M from its own metrics; it needs the side material
        for (int k = 0; k < n; ++k) {
          S.normal[k] = B.curve[s].n1[k];
          S.normal[k + n] = B.curve[s].n2[k];
        }
        if (B.heterogeneous) {
          B.side_mat[s].resize((size_t)n * 3);
          for (int k = 0; k < n; ++k) {
            int i = s == 0 ? B.mgx : (s == 1 ? B.pgx : B.mgx + k);
            int j = s == 2 ? B.mgy : (s == 3 ? B.pgy : B.mgy + k);
            size_t g = gidx(d, i, j);
            B.side_mat[s][k] = dom.rho[g];
            B.side_mat[s][k + n] = dom.cs[g];
            B.side_mat[s][k + 2 * (size_t)n] = dom.cp[g];
          }
        }
        continue;
      }
      S.M.assign((size_t)n * 5, 1e40);
      for (int k = 0; k < n; ++k) {
        S.normal[k] = B.curve[s].n1[k];
        S.normal[k + n] = B.curve[s].n2[k];
        int i, j;
        if (s == 0) { i = B.mgx; j = B.mgy + k; }
        else if (s == 1) { i = B.pgx; j = B.mgy + k; }
        else if (s == 2) { i = B.mgx + k; j = B.mgy; }
        else { i = B.mgx + k; j = B.pgy; }
        size_t g = gidx(d, i, j);
        double rho, cs, cp;
        if (B.heterogeneous) { rho = dom.rho[g]; cs = dom.cs[g]; cp = dom.cp[g]; }
        else { rho = B.rho; cs = B.cs; cp = B.cp; }
        double mag = (s < 2) ? std::sqrt(dom.xr[g] * dom.xr[g] + dom.yr[g] * dom.yr[g])
                             : std::sqrt(dom.xq[g] * dom.xq[g] + dom.yq[g] * dom.yq[g]);
        fdmap::edge_impedances(rho, cs, cp, mag, dom.J[g], op.H00i, &S.M[k], n);
      }
    }
  }

  // ---- source (init_source + search in set_source, source.f90:21-145, 181-204)
  Namelist sl = read_nml(text, 0, "source_list");
  fdmap_source& src = d.src;
  src.gx = get_real(sl, "gx", 0); src.gy = get_real(sl, "gy", 0); src.gz = get_real(sl, "gz", 0);
  src.x0 = get_real(sl, "x0", 0); src.y0 = get_real(sl, "y0", 0);
  src.t_duration = get_real(sl, "t_duration", 1.0); src.t_center = get_real(sl, "t_center", 0.0);
  src.Fx = get_real(sl, "fx", 0); src.Fy = get_real(sl, "fy", 0); src.Fz = get_real(sl, "fz", 0);
  src.Mxx = get_real(sl, "mxx", 0); src.Mxy = get_real(sl, "mxy", 0); src.Myy = get_real(sl, "myy", 0);
  src.Mzx = get_real(sl, "mzx", 0); src.Mzy = get_real(sl, "mzy", 0);
  src.stf = stf_code(get_str(sl, "source_time_function", "gaussian"));
  {
    // tsunami forcing and forcing from file (source.f90:41-115, 299-322)
    const std::string sproblem = get_str(sl, "problem", "");
    if (sproblem == "Forcing") src.gauss_forcing = 1;
    else if (sproblem != "") fail(FDMAP_ERR_UNSUPPORTED, "source problem '" + sproblem + "' is not supported");
    src.gauss_amp = get_real(sl, "gauss_amp", 0.0);
    src.gauss_sigma = get_real(sl, "gauss_sigma", 0.0);
    src.gauss_sigmat = get_real(sl, "gauss_sigmat", 0.0);
    if (get_bool(sl, "forcing_from_file", false)) {
      dom.forcing_path = join_path(base, get_str(sl, "forcing_filename", ""));
      src.forcing_filename = dom.forcing_path.c_str();
    }
  }
  src.use_gravity = (src.gx != 0 || src.gy != 0 || src.gz != 0);
  src.use_singular = (src.Fx != 0 || src.Fy != 0 || src.Fz != 0) ||
                     (src.Mxx != 0 || src.Mxy != 0 || src.Myy != 0 || src.Mzx != 0 || src.Mzy != 0);

  // ---- block descriptors
  dom.blocks.resize(nblocks);
  for (int b = 0; b < nblocks; ++b) {
    BlockIn& B = dom.bin[b];
    fdmap_block& fb = dom.blocks[b];
    fb.mgx = B.mgx; fb.pgx = B.pgx; fb.mgy = B.mgy; fb.pgy = B.pgy;
    fb.rho = B.rho; fb.cs = B.cs; fb.cp = B.cp; fb.G = B.G; fb.M = B.M; fb.gamma = B.gamma; fb.nu = B.nu;
    fb.Cdiss = B.Cdiss;
    fb.pmlx = B.pmlx ? 1 : 0; fb.pmly = B.pmly ? 1 : 0;
    fb.pml_n = B.pml_n; fb.pml_sigma = B.pml_sigma; fb.pml_kappa = B.pml_kappa;
    fb.pml_mx = B.pml_mx; fb.pml_px = B.pml_px; fb.pml_my = B.pml_my; fb.pml_py = B.pml_py;
    // a PML block of a heterogeneous medium runs the PML rates with the
    // block's homogeneous material, as set_rates does (time_step.f90:354-420
    // come before the heterogeneous branch); szz keeps the node's nu (486-490)
    for (int q = 0; q < 9; ++q) fb.F0[q] = B.F0v[q];
    for (int s = 0; s < 4; ++s) {
      fdmap_side& fs = fb.side[s];
      fs.bc = B.bc[s];
      fs.n = (s < 2) ? B.ny : B.nx;
      fs.M = B.side[s].M.data();
      fs.F0 = B.side[s].F0.data();
      fs.normal = B.side[s].normal.data();
      fs.x = B.side[s].x.data();
      fs.y = B.side[s].y.data();
    }
    fb.src_ok = 0;
    if (src.use_singular) {
      // the search reads the bottom row of x and the left column of y only
      // (interpolated here when the device builds the body)
      std::vector<double> xs(B.nx), ys(B.ny);
      for (int i = B.mgx; i <= B.pgx; ++i) xs[i - B.mgx] = dev_body ? node_coord(B, i, B.mgy, 0) : dom.x[gidx(d, i, B.mgy)];
      for (int j = B.mgy; j <= B.pgy; ++j) ys[j - B.mgy] = dev_body ? node_coord(B, B.mgx, j, 1) : dom.y[gidx(d, B.mgx, j)];
      bool outx, outy;
      int i0 = search_floor(xs.data(), B.nx, src.x0, &outx) + B.mgx - 1;
      int j0 = search_floor(ys.data(), B.ny, src.y0, &outy) + B.mgy - 1;
      if (!outx && !outy) {
        fb.src_ok = 1;
        fb.src_i0 = i0; fb.src_j0 = j0;
        fb.src_hx = xs[1] - xs[0];
        fb.src_hy = ys[1] - ys[0];
        fb.src_ax = (src.x0 - xs[i0 - B.mgx]) / fb.src_hx;
        fb.src_ay = (src.y0 - ys[j0 - B.mgy]) / fb.src_hy;
      }
    }
  }

  // ---- time step (set_dt, domain.f90:1462-1535)
  double cmax;
  {
    double cs = 0, cp = 0;
    if (any_het) {
      cs = -HUGE_VAL; cp = -HUGE_VAL;
      for (size_t g = 0; g < NN; ++g) { cs = std::max(cs, dom.cs[g]); cp = std::max(cp, dom.cp[g]); }
    } else {
      for (auto& B : dom.bin) { cs = std::max(cs, B.cs); cp = std::max(cp, B.cp); }
    }
    cmax = std::sqrt(cs * cs + cp * cp);
  }
  d.t0 = t0;
  if (dev_body) {
    // finished by fdmap_host_set_spacing once the device has reduced hmin, hmax
    dom.body.dt_in = dt; dom.body.CFL_in = CFL; dom.body.refine = refine; dom.body.tend = tend;
    dom.body.nt_in = nt; dom.body.c = cmax;
    for (int b = 0; b < nblocks; ++b) dom.bbody[b].Cdiss = dom.bin[b].Cdiss;
    dom.body.blocks = dom.bbody.data();
    d.dt = NAN; d.CFL = NAN; d.nt = 0; d.hmin = NAN; d.hmax = NAN;
    for (int b = 0; b < nblocks; ++b) dom.blocks[b].Cdiss = 0.0;
  } else {
    if (hmin <= 0.0) fail(FDMAP_ERR_INVALID_ARG, "Minimum grid spacing must be positive");
    fdmap::finish_time_step(dt, CFL, refine, tend, nt, cmax, hmin, &dt, &CFL, &nt);
    d.dt = dt; d.CFL = CFL; d.nt = nt; d.hmin = hmin; d.hmax = hmax;
    // artificial dissipation scaled as (wave speed)/(grid spacing) (domain.f90:317-320)
    for (int b = 0; b < nblocks; ++b) {
      BlockIn& B = dom.bin[b];
      B.Cdiss = B.Cdiss * CFL / dt;
      dom.blocks[b].Cdiss = B.Cdiss;
    }
  }

  // ---- interfaces (get_iface_neighbors, init_iface, init_iface_blocks, init_friction,
  //      init_thermpres; domain.f90:1648-1682, interfaces.f90:26-278, friction.f90:55-317)
  std::vector<int> Im(nifaces), Ip(nifaces), dir(nifaces);
  {
    for (int ix = 1; ix <= nbx - 1; ++ix)
      for (int iy = 1; iy <= nby; ++iy) {
        int k = ix + (iy - 1) * (nbx - 1) - 1;
        Im[k] = ix + nbx * (iy - 1); Ip[k] = ix + 1 + nbx * (iy - 1); dir[k] = 0;
      }
    int off = (nbx - 1) * nby;
    for (int ix = 1; ix <= nbx; ++ix)
      for (int iy = 1; iy <= nby - 1; ++iy) {
        int k = off + ix + (iy - 1) * nbx - 1;
        Im[k] = ix + nbx * (iy - 1); Ip[k] = ix + nbx * iy; dir[k] = 1;
      }
  }
  dom.ifaces.resize(nifaces);
  dom.istore.resize(nifaces);
  for (int k = 0; k < nifaces; ++k) {
    fdmap_iface& I = dom.ifaces[k];
    IfaceStore& IS = dom.istore[k];
    size_t mk = seek_marker(text, "!---IFACE" + std::to_string(k + 1) + "---");
    Namelist il = read_nml(text, mk, "interface_list");
    std::string coupling = get_str(il, "coupling", "locked");
    int iblockm = get_int(il, "iblockm", Im[k]), iblockp = get_int(il, "iblockp", Ip[k]);
    std::string direction = get_str(il, "direction", dir[k] == 0 ? "x" : "y");
    int mg = get_int(il, "mg", 0), pg = get_int(il, "pg", 0);
    const BlockIn& Gm = dom.bin[iblockm - 1];
    const BlockIn& Gp = dom.bin[iblockp - 1];
    I.direction = (direction == "x") ? 0 : 1;
    if (mg == 0 || pg == 0) {
      if (I.direction == 0) { mg = Gm.mgy; pg = Gm.pgy; } else { mg = Gm.mgx; pg = Gm.pgx; }
    } else {
      int ib = I.direction == 0 ? Gm.iblock_y : Gm.iblock_x;
      if (mg == pg) { mg = (int)std::ceil((double)(mg - ib) * refine) + ib; pg = mg; }
      else {
        mg = (int)std::ceil((double)(mg - ib) * refine) + ib;
        pg = (int)std::ceil((double)(pg - ib) * refine) + ib;
      }
    }
    int m, p;
    if (I.direction == 0) { m = std::max(Gm.mgy, Gp.mgy); p = std::min(Gm.pgy, Gp.pgy); }
    else { m = std::max(Gm.mgx, Gp.mgx); p = std::min(Gm.pgx, Gp.pgx); }
    I.m = std::max(mg, m);
    I.p = std::min(pg, p);
    if (I.p < I.m) fail(FDMAP_ERR_INVALID_ARG, "interface " + std::to_string(k + 1) + " has no nodes");
    I.iblockm = iblockm - 1;
    I.iblockp = iblockp - 1;
    if (coupling == "locked") I.coupling = FDMAP_COUPLING_LOCKED;
    else if (coupling == "friction") I.coupling = FDMAP_COUPLING_FRICTION;
    else fail(FDMAP_ERR_UNSUPPORTED, "interface coupling '" + coupling + "' is not supported");
    int n = I.p - I.m + 1;
    // geometry from the minus block's side (R for 'x', T for 'y')
    int sm = I.direction == 0 ? 1 : 2 + 1;
    int off = I.direction == 0 ? Gm.mgy : Gm.mgx;
    IS.x.resize(n); IS.y.resize(n); IS.nhat.resize(2 * (size_t)n);
    for (int q = 0; q < n; ++q) {
      int kk = I.m + q - off;
      IS.x[q] = Gm.curve[sm].x[kk];
      IS.y[q] = Gm.curve[sm].y[kk];
      IS.nhat[q] = Gm.curve[sm].n1[kk];
      IS.nhat[q + n] = Gm.curve[sm].n2[kk];
    }
    I.x = IS.x.data(); I.y = IS.y.data(); I.nhat = IS.nhat.data();
    fdmap_friction& fr = I.fr;
    fr = fdmap_friction{};
    if (I.coupling != FDMAP_COUPLING_FRICTION) continue;
    if (mk == std::string::npos) fail(FDMAP_ERR_INVALID_ARG, "String '!---IFACE" + std::to_string(k + 1) + "---' not found in file");
    Namelist fl = read_nml(text, mk, "friction_list");
    std::string law = get_str(fl, "friction_law", "frictionless");
    fr.law = law_code(law);
    if (get_str(fl, "problem", "") != "") fail(FDMAP_ERR_UNSUPPORTED, "friction problem presets are not supported");
    fr.force = get_bool(fl, "force", false) ? 1 : 0;
    fr.angle = 0.017453292519943 * get_real(fl, "angle", 0.0);
    fr.kn_c0 = get_real(fl, "kn", 0.0, "kinematic", "c0");
    fr.kn_fd = get_real(fl, "kn", 0.0, "kinematic", "fd");
    fr.kn_dfdx = get_real(fl, "kn", 1.0, "kinematic", "dfdx");
    fr.kn_vL = get_real(fl, "kn", 0.0, "kinematic", "vl");
    fr.kn_vR = get_real(fl, "kn", 0.0, "kinematic", "vr");
    fr.kn_xL = get_real(fl, "kn", 0.0, "kinematic", "xl");
    fr.kn_xR = get_real(fl, "kn", 0.0, "kinematic", "xr");
    fr.kn_tmax = get_real(fl, "kn", HUGE_VAL, "kinematic", "tmax");
    fr.ld_shape = ld_code(get_str(fl, "ld", "smooth", "load", "shape"));
    fr.ld_S = get_real(fl, "ld", 0.0, "load", "s");
    fr.ld_N = get_real(fl, "ld", 0.0, "load", "n");
    fr.ld_T = get_real(fl, "ld", 0.0, "load", "t");
    fr.ld_R = get_real(fl, "ld", 1.0, "load", "r");
    fr.ld_x0 = get_real(fl, "ld", 0.0, "load", "x0");
    fr.ld_y0 = get_real(fl, "ld", 0.0, "load", "y0");
    std::string rupf = get_str(fl, "rup_field", "V");
    if (rupf == "V") fr.rup_field = 0;
    else if (rupf == "D") fr.rup_field = 1;
    else fail(FDMAP_ERR_INVALID_ARG, "Invalid field to define rupture front");
    fr.rup_threshold = get_real(fl, "rup_threshold", 0.0);
    fr.xlockm = get_real(fl, "xlockm", -1e10);
    fr.xlockp = get_real(fl, "xlockp", 1e10);
    fr.flock = get_real(fl, "flock", 1e10);
    fr.skempton = get_real(fl, "skempton", 0.0);
    fr.reg = get_bool(fl, "reg", false) ? 1 : 0;
    double Psi0 = get_real(fl, "psi0", 0.0);
    FrictionStore& FS = IS.fr;
    auto fill = [n](std::vector<double>& v, double val) { v.assign(n, val); };
    fill(FS.V, 1e40); fill(FS.O, 1e40); fill(FS.S, 1e40); fill(FS.N, 1e40); fill(FS.S0, 1e40); fill(FS.N0, 1e40);
    fill(FS.Ds, 0); fill(FS.Dn, 0); fill(FS.DDs, 0); fill(FS.DDn, 0);
    fill(FS.Psi, Psi0); fill(FS.DPsi, 1e40); fill(FS.D, 0); fill(FS.trup, 1e10);
    fill(FS.W, 0); fill(FS.DW, 1e40); fill(FS.Nreg, 1e40); fill(FS.DNreg, 1e40);
    double rs_c[7] = {get_real(fl, "rs", 0.01, "ratestate_constant", "a"), get_real(fl, "rs", 0.014, "ratestate_constant", "b"),
                      get_real(fl, "rs", 1e-6, "ratestate_constant", "v0"), get_real(fl, "rs", 0.6, "ratestate_constant", "f0"),
                      get_real(fl, "rs", 0.4, "ratestate_constant", "l"), get_real(fl, "rs", 0.2, "ratestate_constant", "fw"),
                      get_real(fl, "rs", 1e20, "ratestate_constant", "vw")};
    double sw_c[4] = {get_real(fl, "sw", 0.0, "slipweak_constant", "c0"), get_real(fl, "sw", 1.0, "slipweak_constant", "fs"),
                      get_real(fl, "sw", 0.0, "slipweak_constant", "fd"), get_real(fl, "sw", 1.0, "slipweak_constant", "dc")};
    bool is_rs = fr.law >= FDMAP_FR_SL;
    if (is_rs) {
      fill(FS.a, rs_c[0]); fill(FS.b, rs_c[1]); fill(FS.V0, rs_c[2]); fill(FS.f0, rs_c[3]);
      fill(FS.L, rs_c[4]); fill(FS.fw, rs_c[5]); fill(FS.Vw, rs_c[6]);
    } else if (fr.law == FDMAP_FR_SW) {
      fill(FS.c0, sw_c[0]); fill(FS.fs, sw_c[1]); fill(FS.fd, sw_c[2]); fill(FS.Dc, sw_c[3]);
    }
    // per-interface files hold (pg-mg+1) values per array; this process reads m..p
    int ntot = pg - mg + 1;
    size_t skip = (size_t)(I.m - mg);
    auto read_arrays = [&](const std::string& fname, std::vector<std::vector<double>*> arrs) {
      std::vector<double> v = read_binary_doubles(join_path(base, fname), (size_t)ntot * arrs.size());
      for (size_t a = 0; a < arrs.size(); ++a)
        arrs[a]->assign(v.begin() + a * ntot + skip, v.begin() + a * ntot + skip + n);
    };
    if (get_bool(fl, "friction_file", false)) {
      std::string fname = get_str(fl, "filename", "");
      if (is_rs) read_arrays(fname, {&FS.a, &FS.b, &FS.V0, &FS.f0, &FS.L, &FS.fw, &FS.Vw});
      else if (fr.law == FDMAP_FR_SW) read_arrays(fname, {&FS.c0, &FS.fs, &FS.fd, &FS.Dc});
    }
    if (get_bool(fl, "stress_file", false)) read_arrays(get_str(fl, "stress_filename", ""), {&FS.bsS0, &FS.bsN0});
    if (get_bool(fl, "strength_file", false)) fail(FDMAP_ERR_UNSUPPORTED, "strength_file is not supported");
    if (get_bool(fl, "state_file", false)) read_arrays(get_str(fl, "state_filename", ""), {&FS.Psi});
    Namelist tl = read_nml(text, mk, "thermpres_list");
    fr.tp_use = get_int(tl, "n", 0) != 0 ? 1 : 0;
    fr.tp_p0 = get_real(tl, "p0", 0.0);
    auto ptr = [](std::vector<double>& v) -> double* { return v.empty() ? nullptr : v.data(); };
    fr.a = ptr(FS.a); fr.b = ptr(FS.b); fr.V0 = ptr(FS.V0); fr.f0 = ptr(FS.f0); fr.L = ptr(FS.L);
    fr.fw = ptr(FS.fw); fr.Vw = ptr(FS.Vw);
    fr.c0 = ptr(FS.c0); fr.fs = ptr(FS.fs); fr.fd = ptr(FS.fd); fr.Dc = ptr(FS.Dc);
    fr.bsS0 = ptr(FS.bsS0); fr.bsN0 = ptr(FS.bsN0);
    fr.V = ptr(FS.V); fr.O = ptr(FS.O); fr.S = ptr(FS.S); fr.N = ptr(FS.N); fr.S0 = ptr(FS.S0); fr.N0 = ptr(FS.N0);
    fr.Ds = ptr(FS.Ds); fr.Dn = ptr(FS.Dn); fr.DDs = ptr(FS.DDs); fr.DDn = ptr(FS.DDn);
    fr.Psi = ptr(FS.Psi); fr.DPsi = ptr(FS.DPsi); fr.D = ptr(FS.D); fr.trup = ptr(FS.trup);
    fr.W = ptr(FS.W); fr.DW = ptr(FS.DW); fr.Nreg = ptr(FS.Nreg); fr.DNreg = ptr(FS.DNreg);
  }

  // ---- wire the descriptor
  d.blocks = dom.blocks.data();
  d.ifaces = dom.ifaces.data();
  d.heterogeneous = any_het ? 1 : 0;
  dom.dev_body = dev_body;
  if (dev_body) {
    // body arrays and side impedances come from the device
    for (int b = 0; b < nblocks; ++b)
      for (int s = 0; s < 4; ++s) {
        dom.blocks[b].side[s].M = nullptr;
        dom.bbody[b].side_mat[s] = dom.bin[b].side_mat[s].empty() ? nullptr : dom.bin[b].side_mat[s].data();
      }
    for (int b = 0; b < nblocks; ++b)
      for (int c = 0; c < 2; ++c) {
        dom.bbody[b].LB[c] = dom.bin[b].LB[c]; dom.bbody[b].LT[c] = dom.bin[b].LT[c];
        dom.bbody[b].RB[c] = dom.bin[b].RB[c]; dom.bbody[b].RT[c] = dom.bin[b].RT[c];
      }
    d.body = &dom.body;
  } else {
    d.F = dom.F.data(); d.DF = dom.DF.data();
    d.x = dom.x.data(); d.y = dom.y.data();
    d.xq = dom.xq.data(); d.xr = dom.xr.data(); d.yq = dom.yq.data(); d.yr = dom.yr.data();
    d.J = dom.J.data(); d.Ji = dom.Ji.data();
  }
  if (any_het) {
    d.rho = dom.rho.data(); d.cs = dom.cs.data(); d.cp = dom.cp.data(); d.G = dom.G.data();
    d.M = dom.M.data(); d.gamma = dom.gamma.data(); d.nu = dom.nu.data();
  }
}

}  // namespace

extern "C" int fdmap_host_init(const char* input_text, const char* base_dir, fdmap_domain** out) {
  return fdmap_host_init_ex(input_text, base_dir, 0, out);
}

extern "C" int fdmap_host_init_ex(const char* input_text, const char* base_dir, int flags, fdmap_domain** out) {
  if (!input_text || !out) { g_last_error = "null argument"; return FDMAP_ERR_INVALID_ARG; }
  if (flags & ~FDMAP_INIT_BODY_ON_DEVICE) { g_last_error = "unknown initialisation flags"; return FDMAP_ERR_INVALID_ARG; }
  *out = nullptr;
  std::unique_ptr<fdmap_domain> dom(new (std::nothrow) fdmap_domain());
  if (!dom) { g_last_error = "out of memory"; return FDMAP_ERR_NOMEM; }
  try {
    build(*dom, std::string(input_text), base_dir ? std::string(base_dir) : std::string(),
          (flags & FDMAP_INIT_BODY_ON_DEVICE) != 0);
  } catch (const InitError& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "out of memory";
    return FDMAP_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return FDMAP_ERR_INVALID_ARG;
  }
  g_last_error.clear();
  *out = dom.release();
  return FDMAP_OK;
}

extern "C" int fdmap_host_set_spacing(fdmap_domain* dom, double hmin, double hmax) {
  if (!dom || !dom->dev_body) { g_last_error = "the domain's body was not left to the device"; return FDMAP_ERR_INVALID_ARG; }
  if (!(hmin > 0.0)) { g_last_error = "Minimum grid spacing must be positive"; return FDMAP_ERR_INVALID_ARG; }
  fdmap_desc& d = dom->desc;
  const fdmap_body& bd = dom->body;
  double dt, CFL;
  int nt;
  fdmap::finish_time_step(bd.dt_in, bd.CFL_in, bd.refine, bd.tend, bd.nt_in, bd.c, hmin, &dt, &CFL, &nt);
  d.dt = dt; d.CFL = CFL; d.nt = nt; d.hmin = hmin; d.hmax = hmax;
  for (int b = 0; b < d.nblocks; ++b) dom->blocks[b].Cdiss = dom->bbody[b].Cdiss * CFL / dt;
  return FDMAP_OK;
}

extern "C" const fdmap_desc* fdmap_host_desc(const fdmap_domain* dom) { return dom ? &dom->desc : nullptr; }
extern "C" fdmap_desc* fdmap_host_desc_mut(fdmap_domain* dom) { return dom ? &dom->desc : nullptr; }
extern "C" void fdmap_host_free(fdmap_domain* dom) { delete dom; }
extern "C" const char* fdmap_host_last_error(void) { return g_last_error.c_str(); }

extern "C" int fdmap_host_info(const fdmap_domain* dom, int* ints, double* dbls) {
  if (!dom) return FDMAP_ERR_INVALID_ARG;
  const fdmap_desc& d = dom->desc;
  if (ints) {
    ints[0] = d.mode; ints[1] = d.nF; ints[2] = d.nx; ints[3] = d.ny;
    ints[4] = d.nblocks; ints[5] = d.nifaces; ints[6] = d.nt; ints[7] = d.rk_order;
    ints[8] = d.fd_method; ints[9] = d.heterogeneous;
  }
  if (dbls) {
    dbls[0] = d.t0; dbls[1] = d.dt; dbls[2] = d.CFL; dbls[3] = d.hmin; dbls[4] = d.hmax;
  }
  return FDMAP_OK;
}

extern "C" int fdmap_host_body_flags(const fdmap_domain* dom, int* flags) {
  if (!dom || !flags) return FDMAP_ERR_INVALID_ARG;
  flags[0] = dom->desc.displacement;
  flags[1] = dom->desc.peak;
  flags[2] = dom->desc.energy_balance;
  return FDMAP_OK;
}

extern "C" int fdmap_host_iface_n(const fdmap_domain* dom, int iface) {
  if (!dom || iface < 0 || iface >= dom->desc.nifaces) return FDMAP_ERR_INVALID_ARG;
  return dom->desc.ifaces[iface].p - dom->desc.ifaces[iface].m + 1;
}

extern "C" int fdmap_host_iface_info(const fdmap_domain* dom, int iface, int* info) {
  if (!dom || !info || iface < 0 || iface >= dom->desc.nifaces) return FDMAP_ERR_INVALID_ARG;
  const fdmap_iface& I = dom->desc.ifaces[iface];
  info[0] = I.direction; info[1] = I.m; info[2] = I.p; info[3] = I.coupling;
  return FDMAP_OK;
}

extern "C" int fdmap_host_iface_blocks(const fdmap_domain* dom, int iface, int* blocks) {
  if (!dom || !blocks || iface < 0 || iface >= dom->desc.nifaces) return FDMAP_ERR_INVALID_ARG;
  const fdmap_iface& I = dom->desc.ifaces[iface];
  blocks[0] = I.iblockm; blocks[1] = I.iblockp;
  return FDMAP_OK;
}

extern "C" const double* fdmap_host_iface_xy(const fdmap_domain* dom, int iface, int which) {
  if (!dom || iface < 0 || iface >= dom->desc.nifaces) return nullptr;
  const fdmap_iface& I = dom->desc.ifaces[iface];
  return which == 0 ? I.x : I.y;
}

extern "C" const double* fdmap_host_side_array(const fdmap_domain* dom, int block, int side, const char* name,
                                               long long* count) {
  if (!dom || !name || block < 0 || block >= dom->desc.nblocks || side < 0 || side > 3) return nullptr;
  const fdmap_side& S = dom->desc.blocks[block].side[side];
  const std::string n = name;
  const double* p = nullptr;
  long long len = 0;
  if (n == "F0") { p = S.F0; len = (long long)S.n * dom->desc.nF; }
  else if (n == "M") { p = S.M; len = (long long)S.n * 5; }
  else if (n == "normal") { p = S.normal; len = (long long)S.n * 2; }
  else if (n == "x") { p = S.x; len = S.n; }
  else if (n == "y") { p = S.y; len = S.n; }
  if (p && count) *count = len;
  return p;
}

extern "C" double fdmap_host_block_cdiss(const fdmap_domain* dom, int block) {
  if (!dom || block < 0 || block >= dom->desc.nblocks) return FDMAP_ERR_INVALID_ARG;
  return dom->desc.blocks[block].Cdiss;
}

extern "C" int fdmap_host_block_pml(const fdmap_domain* dom, int block, int* flags, double* params) {
  if (!dom || block < 0 || block >= dom->desc.nblocks) return FDMAP_ERR_INVALID_ARG;
  const fdmap_block& b = dom->desc.blocks[block];
  if (flags) { flags[0] = b.pmlx; flags[1] = b.pmly; }
  if (params) {
    params[0] = b.pml_n; params[1] = b.pml_sigma; params[2] = b.pml_kappa;
    params[3] = b.pml_mx; params[4] = b.pml_px; params[5] = b.pml_my; params[6] = b.pml_py;
  }
  return FDMAP_OK;
}

extern "C" int fdmap_host_block_limits(const fdmap_domain* dom, int block, int* lim) {
  if (!dom || !lim || block < 0 || block >= dom->desc.nblocks) return FDMAP_ERR_INVALID_ARG;
  const fdmap_block& b = dom->desc.blocks[block];
  lim[0] = b.mgx; lim[1] = b.pgx; lim[2] = b.mgy; lim[3] = b.pgy;
  return FDMAP_OK;
}

extern "C" double* fdmap_host_array(fdmap_domain* dom, const char* name, long long* count) {
  if (!dom || !name) return nullptr;
  std::string n(name);
  std::vector<double>* v = nullptr;
  if (n == "F") v = &dom->F;
  else if (n == "DF") v = &dom->DF;
  else if (n == "x") v = &dom->x;
  else if (n == "y") v = &dom->y;
  else if (n == "xq") v = &dom->xq;
  else if (n == "xr") v = &dom->xr;
  else if (n == "yq") v = &dom->yq;
  else if (n == "yr") v = &dom->yr;
  else if (n == "J") v = &dom->J;
  else if (n == "Ji") v = &dom->Ji;
  else if (n == "rho") v = &dom->rho;
  else if (n == "cs") v = &dom->cs;
  else if (n == "cp") v = &dom->cp;
  else if (n == "G") v = &dom->G;
  else if (n == "M") v = &dom->M;
  else if (n == "gamma") v = &dom->gamma;
  else if (n == "nu") v = &dom->nu;
  if (!v || v->empty()) return nullptr;
  if (count) *count = (long long)v->size();
  return v->data();
}
