// udf_reader.cpp -- KAPSEL's UDF input and record files read from C or C++.
//
// The reference reads its input through OCTA's UDFManager
// (Gourmet_file_io, input.cxx:438-1818), a library that is not part of the
// reference.  A UDF file holds definition blocks (\begin{def} or
// \begin{global_def}, possibly pulled in by \include{"define.udf"}) that
// declare classes and named entries with types, and \begin{data} blocks
// whose values are positional: a struct is {v1, v2, ...} in declaration
// order, an array is [e0, e1, ...], a select is a string.  This reader pairs
// each value with its declared type and flattens every data block into the
// dotted paths the reference asks for, e.g. constitutive_eq.Navier_Stokes.DX
// or object_type.spherical_particle.Particle_spec[0].Particle_number; an
// output file (Output_udf, one data block per record) gives one flattened
// record per block.  kapsel_udf_to_params then derives the library's
// kapsel_params as Gourmet_file_io and Set_global_parameters do (including
// the automatic time step, input.cxx:316-362).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kapsel_gpu.h"

namespace {

struct UdfError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

enum TokKind { T_STR, T_NUM, T_NAME, T_PUNCT, T_CMD };
struct Tok {
  TokKind kind;
  std::string text;
};

bool name_start(char c) { return std::isalpha((unsigned char)c) || c == '_'; }
bool name_char(char c) { return std::isalnum((unsigned char)c) || c == '_'; }

// A number as the token pattern [-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)? not
// followed by a name character; returns its length or 0.
size_t match_number(const std::string &s, size_t p) {
  size_t i = p;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) ++i;
  size_t digits = 0;
  while (i < s.size() && std::isdigit((unsigned char)s[i])) ++i, ++digits;
  if (digits > 0) {
    if (i < s.size() && s[i] == '.') {
      ++i;
      while (i < s.size() && std::isdigit((unsigned char)s[i])) ++i;
    }
  } else {
    if (i < s.size() && s[i] == '.') {
      ++i;
      size_t frac = 0;
      while (i < s.size() && std::isdigit((unsigned char)s[i])) ++i, ++frac;
      if (frac == 0) return 0;
    } else {
      return 0;
    }
  }
  if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
    size_t j = i + 1;
    if (j < s.size() && (s[j] == '+' || s[j] == '-')) ++j;
    size_t ed = 0;
    while (j < s.size() && std::isdigit((unsigned char)s[j])) ++j, ++ed;
    if (ed > 0) i = j;
  }
  if (i < s.size() && name_start(s[i])) return 0;
  return i - p;
}

std::vector<Tok> tokenize(const std::string &s) {
  std::vector<Tok> out;
  size_t p = 0;
  while (p < s.size()) {
    const char c = s[p];
    if (std::isspace((unsigned char)c)) {
      ++p;
    } else if (c == '/' && p + 1 < s.size() && s[p + 1] == '/') {
      while (p < s.size() && s[p] != '\n') ++p;
    } else if (c == '\\' && p + 1 < s.size() && name_start(s[p + 1])) {
      size_t q = p + 1;
      while (q < s.size() && name_char(s[q])) ++q;
      if (q < s.size() && s[q] == '{') {
        const size_t e = s.find('}', q);
        if (e == std::string::npos) throw UdfError("unterminated command");
        out.push_back({T_CMD, s.substr(p, e + 1 - p)});
        p = e + 1;
      } else {
        throw UdfError("unexpected character '\\'");
      }
    } else if (c == '"' || c == '\'') {
      size_t q = p + 1;
      while (q < s.size() && s[q] != c) q += s[q] == '\\' ? 2 : 1;
      if (q >= s.size()) throw UdfError("unterminated string");
      out.push_back({T_STR, s.substr(p, q + 1 - p)});
      p = q + 1;
    } else if (size_t n = match_number(s, p)) {
      out.push_back({T_NUM, s.substr(p, n)});
      p += n;
    } else if (name_start(c)) {
      size_t q = p;
      while (q < s.size() && name_char(s[q])) ++q;
      out.push_back({T_NAME, s.substr(p, q - p)});
      p = q;
    } else if (std::strchr("{}[],:;", c)) {
      out.push_back({T_PUNCT, std::string(1, c)});
      ++p;
    } else {
      throw UdfError(std::string("unexpected character '") + c + "'");
    }
  }
  return out;
}

struct Type;
struct Field {
  std::string name;
  int dims;
  std::shared_ptr<Type> type;
};
struct Type {
  enum Kind { SCALAR, SELECT, STRUCT } kind;
  std::string base;  // double, float, int, string
  std::vector<Field> fields;
};

struct Reader {
  const std::vector<Tok> &t;
  size_t i = 0;
  explicit Reader(const std::vector<Tok> &toks) : t(toks) {}
  bool done() const { return i >= t.size(); }
  const Tok *peek() const { return i < t.size() ? &t[i] : nullptr; }
  const Tok &next() {
    if (i >= t.size()) throw UdfError("unexpected end of block");
    return t[i++];
  }
  void expect(const char *v) {
    const Tok &k = next();
    if (k.text != v) throw UdfError("expected '" + std::string(v) + "', found '" + k.text + "'");
  }
  bool accept(const char *v) {
    if (i < t.size() && t[i].kind != T_STR && t[i].text == v) {
      ++i;
      return true;
    }
    return false;
  }
};

struct Defs {
  std::map<std::string, std::shared_ptr<Type>> classes;
  std::vector<Field> entries;
  const Field *entry(const std::string &n) const {
    for (const Field &f : entries)
      if (f.name == n) return &f;
    return nullptr;
  }
};

std::vector<Field> parse_fields(Reader &r, Defs &d, const char *close);

std::shared_ptr<Type> parse_type(Reader &r, Defs &d) {
  const Tok &k = r.next();
  std::shared_ptr<Type> t;
  if (k.kind == T_PUNCT && k.text == "{") {
    t = std::make_shared<Type>();
    t->kind = Type::STRUCT;
    t->fields = parse_fields(r, d, "}");
  } else if (k.kind == T_NAME && k.text == "select") {
    r.expect("{");
    while (!r.accept("}")) r.next();  // the choices
    t = std::make_shared<Type>();
    t->kind = Type::SELECT;
  } else if (k.kind == T_NAME && (k.text == "double" || k.text == "float" || k.text == "int" || k.text == "string")) {
    t = std::make_shared<Type>();
    t->kind = Type::SCALAR;
    t->base = k.text;
  } else if (k.kind == T_NAME) {
    auto it = d.classes.find(k.text);
    if (it == d.classes.end()) throw UdfError("unknown type '" + k.text + "'");
    t = it->second;
  } else {
    throw UdfError("bad type token '" + k.text + "'");
  }
  while (r.peek() && r.peek()->kind == T_STR) r.next();  // descriptions
  return t;
}

Field parse_field(Reader &r, Defs &d) {
  const Tok &k = r.next();
  if (k.kind != T_NAME) throw UdfError("expected a field name, found '" + k.text + "'");
  Field f;
  f.name = k.text;
  f.dims = 0;
  while (r.accept("[")) {
    r.expect("]");
    ++f.dims;
  }
  r.expect(":");
  f.type = parse_type(r, d);
  return f;
}

std::vector<Field> parse_fields(Reader &r, Defs &d, const char *close) {
  std::vector<Field> out;
  while (!r.accept(close)) {
    if (r.accept(",")) continue;
    out.push_back(parse_field(r, d));
  }
  return out;
}

void add_def_block(const std::string &body, Defs &d) {
  const std::vector<Tok> toks = tokenize(body);
  Reader r(toks);
  while (!r.done()) {
    if (r.accept(",") || r.accept(";")) continue;
    if (r.peek()->kind == T_NAME && r.peek()->text == "class") {
      r.next();
      const std::string name = r.next().text;
      r.expect(":");
      d.classes[name] = parse_type(r, d);
    } else {
      d.entries.push_back(parse_field(r, d));
    }
  }
}

// One flattened value: numbers keep their parsed double and token text.
struct Value {
  std::string path, text;
  double num = 0.0;
  bool is_string = false;
};
using Record = std::vector<Value>;

void parse_value(Reader &r, const Type &t, int dims, const std::string &path, Record &out) {
  if (dims > 0) {
    r.expect("[");
    int n = 0;
    while (!r.accept("]")) {
      if (r.accept(",")) continue;
      parse_value(r, t, dims - 1, path + "[" + std::to_string(n++) + "]", out);
    }
    return;
  }
  if (t.kind == Type::STRUCT) {
    r.expect("{");
    for (const Field &f : t.fields) {
      while (r.accept(",")) {
      }
      parse_value(r, *f.type, f.dims, path + "." + f.name, out);
    }
    while (r.accept(",")) {
    }
    r.expect("}");
    return;
  }
  const Tok &k = r.next();
  Value v;
  v.path = path;
  if (k.kind == T_STR) {
    v.text = k.text.substr(1, k.text.size() - 2);
    v.is_string = true;
  } else if (k.kind == T_NUM) {
    v.num = std::strtod(k.text.c_str(), nullptr);
    if (t.kind == Type::SCALAR && t.base == "int") v.num = std::trunc(v.num);
    v.text = k.text;
  } else if (k.kind == T_NAME) {  // a bare word
    v.text = k.text;
    v.is_string = true;
  } else {
    throw UdfError("expected a value, found '" + k.text + "'");
  }
  out.push_back(v);
}

Record parse_data_block(const std::string &body, const Defs &d) {
  const std::vector<Tok> toks = tokenize(body);
  Reader r(toks);
  Record rec;
  while (!r.done()) {
    if (r.accept(",") || r.accept(";")) continue;
    const Tok &k = r.next();
    int dims = 0;
    while (r.accept("[")) {
      r.expect("]");
      ++dims;
    }
    r.expect(":");
    const Field *f = d.entry(k.text);
    if (!f) throw UdfError("no definition for '" + k.text + "'");
    parse_value(r, *f->type, f->dims, k.text, rec);
  }
  // the flattened path of a top-level entry has no leading dot
  return rec;
}

std::string read_file(const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw UdfError("cannot open " + path);
  std::string s;
  char buf[65536];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
  std::fclose(f);
  return s;
}

std::string dir_of(const std::string &p) {
  const size_t s = p.rfind('/');
  return s == std::string::npos ? std::string(".") : p.substr(0, s);
}

// Walks the top-level \begin{..} ... \end{..} blocks and \include{..} of a
// file in order: definitions are added, data blocks become records.
void parse_text(const std::string &text, const std::string &base, Defs &d, std::vector<Record> *records) {
  int depth = 0;
  size_t start = 0, p = 0;
  std::string name;
  while ((p = text.find('\\', p)) != std::string::npos) {
    size_t q = p + 1;
    while (q < text.size() && std::isalpha((unsigned char)text[q])) ++q;
    const std::string kw = text.substr(p + 1, q - p - 1);
    if ((kw != "begin" && kw != "end" && kw != "include") || q >= text.size() || text[q] != '{') {
      p = q;
      continue;
    }
    const size_t e = text.find('}', q);
    if (e == std::string::npos) break;
    std::string arg = text.substr(q + 1, e - q - 1);
    if (kw == "include" && depth == 0) {
      size_t a = arg.find_first_not_of(" \t\"");
      size_t b = arg.find_last_not_of(" \t\"");
      const std::string file = a == std::string::npos ? std::string() : arg.substr(a, b - a + 1);
      const std::string path = !file.empty() && file[0] == '/' ? file : base + "/" + file;
      parse_text(read_file(path), dir_of(path), d, nullptr);
    } else if (kw == "begin") {
      if (depth == 0) {
        name = arg;
        start = e + 1;
      }
      ++depth;
    } else if (kw == "end") {
      --depth;
      if (depth == 0) {
        const std::string body = text.substr(start, p - start);
        if (name == "def" || name == "global_def")
          add_def_block(body, d);
        else if (name == "data" && records)
          records->push_back(parse_data_block(body, d));
      }
    }
    p = e + 1;
  }
}

}  // namespace

struct kapsel_udf {
  std::vector<Record> records;
  std::vector<std::map<std::string, size_t>> index;
  std::string error;
};

namespace {
const Value *find(const kapsel_udf *u, int record, const char *path) {
  if (!u || record < 0 || record >= (int)u->records.size() || !path) return nullptr;
  auto it = u->index[record].find(path);
  return it == u->index[record].end() ? nullptr : &u->records[record][it->second];
}
double num_or(const kapsel_udf *u, const std::string &path, double dflt, bool *missing = nullptr) {
  const Value *v = find(u, 0, path.c_str());
  if (!v || v->is_string) {
    if (missing) *missing = true;
    return dflt;
  }
  return v->num;
}
std::string str_or(const kapsel_udf *u, const std::string &path, const char *dflt) {
  const Value *v = find(u, 0, path.c_str());
  return v ? v->text : std::string(dflt);
}
}  // namespace

extern "C" {

int kapsel_udf_read(const char *path, kapsel_udf **out) {
  if (!path || !out) return KAPSEL_EINVAL;
  *out = nullptr;
  std::unique_ptr<kapsel_udf> u(new (std::nothrow) kapsel_udf);
  if (!u) return KAPSEL_ENOMEM;
  try {
    Defs d;
    std::string p(path);
    parse_text(read_file(p), dir_of(p), d, &u->records);
  } catch (const std::exception &e) {
    fprintf(stderr, "kapsel_udf_read: %s: %s\n", path, e.what());
    return KAPSEL_EINVAL;
  }
  for (const Record &r : u->records) {
    std::map<std::string, size_t> ix;
    for (size_t i = 0; i < r.size(); ++i) ix[r[i].path] = i;
    u->index.push_back(std::move(ix));
  }
  *out = u.release();
  return 0;
}

int kapsel_udf_destroy(kapsel_udf *u) {
  delete u;
  return 0;
}

int kapsel_udf_records(const kapsel_udf *u) { return u ? (int)u->records.size() : KAPSEL_EINVAL; }

int kapsel_udf_size(const kapsel_udf *u, int record) {
  if (!u || record < 0 || record >= (int)u->records.size()) return KAPSEL_EINVAL;
  return (int)u->records[record].size();
}

int kapsel_udf_entry(const kapsel_udf *u, int record, int i, const char **path, const char **text, int *is_string) {
  if (!u || record < 0 || record >= (int)u->records.size() || i < 0 || i >= (int)u->records[record].size())
    return KAPSEL_EINVAL;
  const Value &v = u->records[record][i];
  if (path) *path = v.path.c_str();
  if (text) *text = v.text.c_str();
  if (is_string) *is_string = v.is_string ? 1 : 0;
  return 0;
}

int kapsel_udf_get_double(const kapsel_udf *u, int record, const char *path, double *value) {
  const Value *v = find(u, record, path);
  if (!v || v->is_string || !value) return KAPSEL_EINVAL;
  *value = v->num;
  return 0;
}

int kapsel_udf_get_string(const kapsel_udf *u, int record, const char *path, const char **text) {
  const Value *v = find(u, record, path);
  if (!v || !text) return KAPSEL_EINVAL;
  *text = v->text.c_str();
  return 0;
}

int kapsel_udf_to_params(const kapsel_udf *u, int precision, kapsel_params *p, double *x, double *q, int *n_user) {
  if (!u || !p || u->records.empty()) return KAPSEL_EINVAL;
  kapsel_params_default(p);
  const std::string eq = str_or(u, "constitutive_eq.type", "");
  if (eq != "Navier_Stokes" && eq != "Electrolyte" && eq != "Shear_Navier_Stokes_Lees_Edwards") return KAPSEL_EINVAL;
  if (str_or(u, "object_type.type", "") != "spherical_particle") return KAPSEL_EINVAL;
  const std::string ps = "object_type.spherical_particle.Particle_spec[0].";
  if (find(u, 0, "object_type.spherical_particle.Particle_spec[1].Particle_number")) return KAPSEL_EINVAL;
  if (str_or(u, ps + "janus_propulsion", "OFF") != "OFF") return KAPSEL_EINVAL;
  const std::string b = "constitutive_eq." + eq + ".";
  bool miss = false;
  p->eq = eq == "Navier_Stokes" ? KAPSEL_EQ_NAVIER_STOKES
          : eq == "Electrolyte" ? KAPSEL_EQ_ELECTROLYTE
                                : KAPSEL_EQ_SHEAR_LE;
  p->precision = precision;
  const char *ax = "XYZ";
  for (int d = 0; d < 3; ++d) p->np_xyz[d] = (int)num_or(u, std::string("mesh.NP") + ax[d], 0, &miss);
  p->dx = num_or(u, b + "DX", 0, &miss);
  p->rho = num_or(u, b + "RHO", 0, &miss);
  p->eta = num_or(u, b + "ETA", 0, &miss);
  p->kbt = num_or(u, b + "kBT", 0, &miss);
  p->alpha_v = num_or(u, b + "alpha_v", eq == "Electrolyte" ? 0.0 : 1.0);
  p->alpha_o = num_or(u, b + "alpha_o", eq == "Electrolyte" ? 0.0 : 1.0);
  p->a = num_or(u, "A", 0, &miss);
  p->a_xi = num_or(u, "A_XI", 0, &miss);
  p->mass_ratio = num_or(u, ps + "MASS_RATIO", 1.0);
  p->n_particles = (int)num_or(u, ps + "Particle_number", 0, &miss);
  p->gravity_g = num_or(u, "gravity.G", 0.0);
  const std::string gd = str_or(u, "gravity.G_direction", "-Z");
  p->gravity_dir = gd == "-X" ? 0 : gd == "-Y" ? 1 : 2;
  p->epsilon = num_or(u, "EPSILON", 1.0);
  const std::string lp = str_or(u, "LJ_powers", "12:6");
  p->lj_powers = lp == "24:12" ? 1 : lp == "36:18" ? 2 : 0;
  const std::string lt = str_or(u, "switch.LJ_truncate", "ON");
  p->lj_truncate = lt == "ON" ? 1 : lt == "OFF" ? 0 : -1;
  p->rotation = str_or(u, "switch.ROTATION", "ON") == "ON" ? 1 : 0;
  const char *xyz = "xyz";
  for (int d = 0; d < 3; ++d)
    p->fix_cell[d] = str_or(u, std::string("switch.FIX_CELL.") + xyz[d], "OFF") == "ON" ? 1 : 0;
  if (eq == "Shear_Navier_Stokes_Lees_Edwards") {
    if (str_or(u, b + "External_field.type", "DC") != "DC") return KAPSEL_EINVAL;
    p->shear_rate = num_or(u, b + "External_field.DC.Shear_rate", 0, &miss);
  }
  if (eq == "Electrolyte") {
    if (str_or(u, b + "Add_salt.type", "") != "salt" || str_or(u, b + "INIT_profile", "") != "Uniform")
      return KAPSEL_EINVAL;
    const std::string s = b + "Add_salt.salt.";
    p->dielectric = num_or(u, b + "Dielectric_cst", 0, &miss);
    p->surface_charge = num_or(u, ps + "Surface_charge", 0, &miss);
    p->debye_length = num_or(u, s + "Debye_length", 0, &miss);
    p->valency_p = num_or(u, s + "Valency_positive_ion", 0, &miss);
    p->valency_n = num_or(u, s + "Valency_negative_ion", 0, &miss);
    p->onsager_p = num_or(u, s + "Onsager_coeff_positive_ion", 0, &miss);
    p->onsager_n = num_or(u, s + "Onsager_coeff_negative_ion", 0, &miss);
    if (str_or(u, b + "Electric_field.type", "OFF") == "ON") {
      if (str_or(u, b + "Electric_field.ON.type", "") != "DC") return KAPSEL_EINVAL;
      for (int d = 0; d < 3; ++d)
        p->e_ext[d] = num_or(u, b + "Electric_field.ON.DC.E" + std::string(1, xyz[d]), 0, &miss);
    }
  }
  // the time step: manual, or DT = factor / (NU KMAX2) with the 2/3-rule
  // KMAX2 (input.cxx:316-362), the Electrolyte taking the ion diffusion
  // time when it is shorter
  if (str_or(u, "time_increment.type", "") == "manual") {
    p->dt = num_or(u, "time_increment.manual.delta_t", 0, &miss);
  } else {
    const double nu = p->eta / p->rho;
    double kmax2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const int n = 1 << p->np_xyz[d];
      const double k = 2.0 * M_PI / (n * p->dx) * ((n + 2) / 3);
      kmax2 += k * k;
    }
    double tdump = 1.0 / (nu * kmax2);
    if (eq == "Electrolyte") {
      const double ons = std::max(p->onsager_p, p->onsager_n);
      tdump = std::min(tdump, 1.0 / (p->kbt * ons * kmax2));
    }
    p->dt = num_or(u, "time_increment.auto.factor", 0, &miss) * tdump;
  }
  if (miss) return KAPSEL_EINVAL;
  int nu = 0;
  if (str_or(u, "switch.INIT_distribution.type", "") == "user_specify") {
    const std::string up = "switch.INIT_distribution.user_specify.Particles[";
    for (int i = 0; i < p->n_particles; ++i) {
      const std::string pre = up + std::to_string(i) + "].";
      for (int d = 0; d < 3; ++d) {
        const double v = num_or(u, pre + "R." + std::string(1, xyz[d]), 0, &miss);
        if (x) x[3 * i + d] = v;
      }
      for (int j = 0; j < 4; ++j) {
        const double v = num_or(u, pre + "q.q" + std::to_string(j), j == 0 ? 1.0 : 0.0);
        if (q) q[4 * i + j] = v;
      }
    }
    if (miss) return KAPSEL_EINVAL;
    nu = p->n_particles;
  }
  if (n_user) *n_user = nu;
  return 0;
}

}  // extern "C"
