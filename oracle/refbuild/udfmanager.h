/*
 * Stand-in for the OCTA GOURMET `UDFManager` / `Location` interface.
 *
 * TEST INFRASTRUCTURE ONLY.  This header lets the unmodified KAPSEL
 * reference sources compile and run as a CPU oracle (oracle/_ref).  The real
 * interface lives in OCTA's libplatform, which is not available; the
 * reference includes it from input.h:21 and uses it in input.cxx:438-1818
 * (Gourmet_file_io), init_particle.cxx:226-288 (user_specify particles),
 * avs_output.cxx:343-450 (Output_udf) and resume.cxx (restart records).
 *
 * The stand-in reads a flat text file of `path = value` lines instead of
 * the positional UDF data format.  Paths are the dotted UDF paths the
 * reference asks for, e.g. `constitutive_eq.Navier_Stokes.DX = 1.0` or
 * `object_type.spherical_particle.Particle_spec[0].Particle_number = 16`.
 * No arithmetic lives behind this interface, only I/O.
 *
 * `put` calls are recorded per record and written by `write()` as
 * `record <n> <path> = <value>` lines (doubles with 17 significant digits),
 * so particle records from Output_udf can be read back by the tests.
 */
#ifndef KAPSEL_ORACLE_UDFMANAGER_STANDIN_H
#define KAPSEL_ORACLE_UDFMANAGER_STANDIN_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

/* The reference sources use `string` unqualified (input.cxx, rigid.h); the
   OCTA header they were written against exports namespace std. */
using namespace std;

class Location {
 public:
  std::string path;
  Location() {}
  Location(const char *p) : path(p) {}
  Location(const std::string &p) : path(p) {}
  std::string sub(const char *s) const { return path.empty() ? std::string(s) : path + "." + s; }
  std::string sub(const std::string &s) const { return sub(s.c_str()); }
  void down(const char *s) { path = sub(s); }
  void down(const std::string &s) { down(s.c_str()); }
  void up() {
    size_t pos = path.rfind('.');
    if (pos == std::string::npos) path.clear(); else path.resize(pos);
  }
  operator std::string() const { return path; }
};

class UDFManager {
 public:
  explicit UDFManager(const char *file) : out_file_(), record_(0) { load(file); }
  UDFManager(const std::string &file) : out_file_(), record_(0) { load(file.c_str()); }
  /* output/restart constructor: (outfile, deffile, flag) */
  template <class T>
  UDFManager(const char *outfile, const char *deffile, T) : out_file_(outfile ? outfile : ""), record_(0) {
    (void)deffile;
  }

  std::string getEngineName() { return lookup_or("engine.name", "kapsel"); }
  std::string getEngineVersion() { return lookup_or("engine.version", "v3.02"); }

  bool get(const std::string &path, std::string &v) {
    const std::string *s = find(path);
    if (!s) return false;
    v = *s;
    return true;
  }
  bool get(const std::string &path, double &v) {
    const std::string *s = find(path);
    if (!s) return false;
    v = strtod(s->c_str(), NULL);
    return true;
  }
  bool get(const std::string &path, float &v) {
    double d;
    if (!get(path, d)) return false;
    v = (float)d;
    return true;
  }
  bool get(const std::string &path, int &v) {
    const std::string *s = find(path);
    if (!s) return false;
    v = (int)strtol(s->c_str(), NULL, 10);
    return true;
  }
  bool get(const std::string &path, unsigned int &v) {
    int i;
    if (!get(path, i)) return false;
    v = (unsigned)i;
    return true;
  }
  bool get(const std::string &path, long &v) {
    const std::string *s = find(path);
    if (!s) return false;
    v = strtol(s->c_str(), NULL, 10);
    return true;
  }
  bool get(const char *path, std::string &v) { return get(std::string(path), v); }
  bool get(const char *path, double &v) { return get(std::string(path), v); }
  bool get(const char *path, int &v) { return get(std::string(path), v); }
  bool get(const Location &l, std::string &v) { return get(l.path, v); }
  bool get(const Location &l, double &v) { return get(l.path, v); }
  bool get(const Location &l, int &v) { return get(l.path, v); }

  /* size("a.b[]") = number of consecutive indices a.b[0], a.b[1], ... present */
  int size(const std::string &path) {
    std::string base = path;
    if (base.size() >= 2 && base.compare(base.size() - 2, 2, "[]") == 0) base.resize(base.size() - 2);
    int n = 0;
    for (;;) {
      char idx[32];
      snprintf(idx, sizeof idx, "[%d]", n);
      std::string prefix = base + idx;
      std::map<std::string, std::string>::const_iterator it = kv_.lower_bound(prefix);
      if (it == kv_.end() || it->first.compare(0, prefix.size(), prefix) != 0) break;
      ++n;
    }
    return n;
  }
  int size(const char *path) { return size(std::string(path)); }

  template <class T>
  void put(const std::string &path, const T &v) { out_.push_back(Entry(record_, path, fmt(v))); }
  template <class T>
  void put(const char *path, const T &v) { put(std::string(path), v); }
  template <class T>
  void put(const Location &l, const T &v) { put(l.path, v); }

  void newRecord() { ++record_; }
  void write() {
    if (out_file_.empty()) return;
    FILE *f = fopen(out_file_.c_str(), "w");
    if (!f) return;
    for (size_t i = 0; i < out_.size(); ++i)
      fprintf(f, "record %d %s = %s\n", out_[i].rec, out_[i].path.c_str(), out_[i].val.c_str());
    fclose(f);
  }

 private:
  struct Entry {
    int rec;
    std::string path, val;
    Entry(int r, const std::string &p, const std::string &v) : rec(r), path(p), val(v) {}
  };
  std::map<std::string, std::string> kv_;
  std::vector<Entry> out_;
  std::string out_file_;
  int record_;

  static std::string fmt(const double &v) { char b[64]; snprintf(b, sizeof b, "%.17g", v); return b; }
  static std::string fmt(const float &v) { return fmt((double)v); }
  static std::string fmt(const int &v) { char b[32]; snprintf(b, sizeof b, "%d", v); return b; }
  static std::string fmt(const unsigned &v) { char b[32]; snprintf(b, sizeof b, "%u", v); return b; }
  static std::string fmt(const long &v) { char b[32]; snprintf(b, sizeof b, "%ld", v); return b; }
  static std::string fmt(const std::string &v) { return v; }
  static std::string fmt(const char *v) { return std::string(v); }

  const std::string *find(const std::string &path) const {
    std::map<std::string, std::string>::const_iterator it = kv_.find(path);
    if (it == kv_.end()) {
      if (getenv("KAPSEL_UDF_TRACE")) fprintf(stderr, "#udf-standin: missing %s\n", path.c_str());
      return NULL;
    }
    return &it->second;
  }
  std::string lookup_or(const char *k, const char *dflt) const {
    const std::string *s = find(k);
    return s ? *s : std::string(dflt);
  }
  static std::string trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n\"");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n\"");
    return s.substr(a, b - a + 1);
  }
  void load(const char *file) {
    FILE *f = fopen(file, "r");
    if (!f) { fprintf(stderr, "#udf-standin: cannot open %s\n", file); exit(EXIT_FAILURE); }
    char line[4096];
    while (fgets(line, sizeof line, f)) {
      std::string s(line);
      /* lines written by write() carry a "record <n> " prefix */
      if (s.compare(0, 7, "record ") == 0) {
        size_t sp = s.find(' ', 7);
        s = sp == std::string::npos ? std::string() : s.substr(sp + 1);
      }
      size_t hash = s.find('#');
      if (hash != std::string::npos) s.resize(hash);
      size_t eq = s.find('=');
      if (eq == std::string::npos) continue;
      std::string k = trim(s.substr(0, eq)), v = trim(s.substr(eq + 1));
      if (!k.empty()) kv_[k] = v;
    }
    fclose(f);
  }
};

#endif
