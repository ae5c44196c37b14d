// he4io.cpp -- namelist, readenc mode 2 and printoutc for the host driver.
#include "he4io.hpp"

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <fstream>
#include <sstream>

namespace he4io {

static std::string lower(std::string s) {
  for (char &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

static std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

// Fortran real literal (d/D exponent allowed) to double
static double to_real(const std::string &tok) {
  std::string t = tok;
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  const double v = strtod(t.c_str(), &end);
  if (end == t.c_str() || *end != 0) throw std::runtime_error("not a real number: '" + tok + "'");
  return v;
}

std::string Namelist::str(const std::string &k, const std::string &dflt) const {
  auto it = values.find(lower(k));
  return it == values.end() ? dflt : it->second;
}

double Namelist::real(const std::string &k, double dflt) const {
  auto it = values.find(lower(k));
  return it == values.end() ? dflt : to_real(it->second);
}

long Namelist::integer(const std::string &k, long dflt) const {
  auto it = values.find(lower(k));
  if (it == values.end()) return dflt;
  char *end = nullptr;
  const long v = strtol(it->second.c_str(), &end, 10);
  if (end == it->second.c_str() || *end != 0) throw std::runtime_error("not an integer: " + k + "=" + it->second);
  return v;
}

bool Namelist::logical(const std::string &k, bool dflt) const {
  auto it = values.find(lower(k));
  if (it == values.end()) return dflt;
  std::string v = lower(it->second);
  if (!v.empty() && v[0] == '.') v = v.substr(1);
  if (!v.empty() && (v[0] == 't')) return true;
  if (!v.empty() && (v[0] == 'f')) return false;
  throw std::runtime_error("not a logical: " + k + "=" + it->second);
}

Namelist parse_namelist(const std::string &text, const std::string &group) {
  Namelist nl;
  nl.group = lower(group);
  // strip comments ('!' to end of line, outside strings)
  std::string s;
  {
    char quote = 0;
    for (size_t i = 0; i < text.size(); i++) {
      const char c = text[i];
      if (quote) {
        s += c;
        if (c == quote) quote = 0;
      } else if (c == '\'' || c == '"') {
        quote = c;
        s += c;
      } else if (c == '!') {
        while (i < text.size() && text[i] != '\n') i++;
        s += '\n';
      } else {
        s += c;
      }
    }
  }
  // find "&group" (or "$group")
  const std::string ls = lower(s);
  size_t pos = std::string::npos;
  for (size_t i = 0; i + 1 + nl.group.size() <= ls.size(); i++) {
    if ((ls[i] == '&' || ls[i] == '$') && ls.compare(i + 1, nl.group.size(), nl.group) == 0) {
      const size_t j = i + 1 + nl.group.size();
      if (j == ls.size() || !(std::isalnum((unsigned char)ls[j]) || ls[j] == '_')) {
        pos = j;
        break;
      }
    }
  }
  if (pos == std::string::npos) throw std::runtime_error("namelist group &" + group + " not found");
  // tokens: name = value(s) [,] ... up to '/' or '&end' outside strings
  size_t i = pos;
  std::string name, value;
  bool in_value = false;
  char quote = 0;
  auto flush = [&]() {
    if (!name.empty()) {
      std::string v = trim(value);
      if (!v.empty() && v.back() == ',') v = trim(v.substr(0, v.size() - 1));
      if (v.size() >= 2 && (v[0] == '\'' || v[0] == '"') && v.back() == v[0]) v = v.substr(1, v.size() - 2);
      nl.values[lower(trim(name))] = v;
    }
    name.clear();
    value.clear();
    in_value = false;
  };
  for (; i < s.size(); i++) {
    const char c = s[i];
    if (quote) {
      value += c;
      if (c == quote) quote = 0;
      continue;
    }
    if (in_value && (c == '\'' || c == '"')) {
      quote = c;
      value += c;
      continue;
    }
    if (c == '/' || (c == '&' && lower(s.substr(i, 4)) == "&end") || (c == '$' && lower(s.substr(i, 4)) == "$end")) {
      flush();
      return nl;
    }
    if (c == '=' && !quote) {
      // the previous token of `value` (after the last separator) is the
      // next variable name when we are inside a value
      if (in_value) {
        std::string v = value;
        size_t k = v.size();
        while (k > 0 && std::isspace((unsigned char)v[k - 1])) k--;
        size_t st = k;
        while (st > 0 && (std::isalnum((unsigned char)v[st - 1]) || v[st - 1] == '_' || v[st - 1] == '(' ||
                          v[st - 1] == ')' || v[st - 1] == ':'))
          st--;
        const std::string next = v.substr(st, k - st);
        value = v.substr(0, st);
        flush();
        name = next;
      }
      in_value = true;
      continue;
    }
    if (in_value)
      value += c;
    else if (!std::isspace((unsigned char)c) && c != ',')
      name += c;
  }
  throw std::runtime_error("namelist &" + group + " is not terminated by '/'");
}

// ---------------------------------------------------------------------------
// list-directed reading
// ---------------------------------------------------------------------------
namespace {

struct ListReader {
  const std::string &s;
  size_t i = 0;
  int repeat = 0;
  std::string pending;

  explicit ListReader(const std::string &str, size_t start) : s(str), i(start) {}

  void skip_sep() {
    while (i < s.size() && (std::isspace((unsigned char)s[i]) || s[i] == ',')) i++;
  }

  std::string raw() {  // one value token (a complex keeps its parentheses)
    if (repeat > 0) {
      repeat--;
      return pending;
    }
    skip_sep();
    if (i >= s.size()) throw std::runtime_error("unexpected end of data");
    size_t st = i;
    if (s[i] == '(') {
      while (i < s.size() && s[i] != ')') i++;
      if (i >= s.size()) throw std::runtime_error("unterminated complex value");
      i++;
    } else {
      while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != ',') {
        if (s[i] == '*') {  // r*value
          const int r = atoi(s.substr(st, i - st).c_str());
          i++;
          const size_t vs = i;
          if (i < s.size() && s[i] == '(') {
            while (i < s.size() && s[i] != ')') i++;
            i++;
          } else {
            while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != ',') i++;
          }
          pending = s.substr(vs, i - vs);
          repeat = r - 1;
          return pending;
        }
        i++;
      }
    }
    return s.substr(st, i - st);
  }

  double real() { return to_real(raw()); }
  long integer() {
    const std::string t = raw();
    char *end = nullptr;
    const long v = strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != 0) throw std::runtime_error("not an integer: '" + t + "'");
    return v;
  }
  std::complex<double> cplx() {
    const std::string t = raw();
    if (t.size() < 5 || t[0] != '(' || t.back() != ')') throw std::runtime_error("not a complex value: '" + t + "'");
    const size_t c = t.find(',');
    if (c == std::string::npos) throw std::runtime_error("not a complex value: '" + t + "'");
    return {to_real(trim(t.substr(1, c - 1))), to_real(trim(t.substr(c + 1, t.size() - c - 2)))};
  }
};

std::string slurp(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::ostringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

// titols: position after the leading lines whose first column is '#'
size_t after_comments(const std::string &s) {
  size_t i = 0;
  while (i < s.size() && s[i] == '#') {
    while (i < s.size() && s[i] != '\n') i++;
    if (i < s.size()) i++;
  }
  return i;
}

// Fortran unformatted sequential records (4-byte length markers)
bool read_record(FILE *f, std::vector<char> *out) {
  int32_t n = 0, m = 0;
  if (fread(&n, 4, 1, f) != 1) return false;
  if (n < 0) throw std::runtime_error("binary record larger than 2 GB is not supported");
  out->resize((size_t)n);
  if (n && fread(out->data(), 1, (size_t)n, f) != (size_t)n) throw std::runtime_error("short binary record");
  if (fread(&m, 4, 1, f) != 1 || m != n) throw std::runtime_error("corrupt binary record marker");
  return true;
}

void write_record(FILE *f, const void *p, size_t n) {
  if (n > 0x7fffffffu) throw std::runtime_error("binary record larger than 2 GB is not supported");
  const int32_t m = (int32_t)n;
  fwrite(&m, 4, 1, f);
  fwrite(p, 1, n, f);
  fwrite(&m, 4, 1, f);
}

bool looks_binary(const std::string &path, int32_t first_record) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("cannot open " + path);
  int32_t n = 0;
  const bool ok = fread(&n, 4, 1, f) == 1;
  fclose(f);
  return ok && n == first_record;
}

}  // namespace

void read_psi(const std::string &path, GridHeader *h, std::vector<std::complex<double>> *psi) {
  if (looks_binary(path, 6 * 8 + 3 * 4)) {
    FILE *f = fopen(path.c_str(), "rb");
    std::vector<char> rec;
    read_record(f, &rec);
    double d[6];
    int32_t n[3];
    memcpy(d, rec.data(), 48);
    memcpy(n, rec.data() + 48, 12);
    h->xmax = d[0], h->ymax = d[1], h->zmax = d[2], h->hx = d[3], h->hy = d[4], h->hz = d[5];
    h->nx = n[0], h->ny = n[1], h->nz = n[2];
    const size_t N = (size_t)h->nx * h->ny * h->nz;
    if (!read_record(f, &rec) || rec.size() != 16 * N) {
      fclose(f);
      throw std::runtime_error(path + ": psi record does not hold nx*ny*nz complex values");
    }
    psi->resize(N);
    memcpy(psi->data(), rec.data(), 16 * N);
    fclose(f);
    return;
  }
  const std::string s = slurp(path);
  ListReader r(s, after_comments(s));
  h->xmax = r.real(), h->ymax = r.real(), h->zmax = r.real();
  h->hx = r.real(), h->hy = r.real(), h->hz = r.real();
  h->nx = (int)r.integer(), h->ny = (int)r.integer(), h->nz = (int)r.integer();
  const size_t N = (size_t)h->nx * h->ny * h->nz;
  psi->resize(N);
  for (size_t k = 0; k < N; k++) (*psi)[k] = r.cplx();
}

void read_density(const std::string &path, GridHeader *h, std::vector<double> *den) {
  const std::string s = slurp(path);
  ListReader r(s, after_comments(s));
  h->xmax = r.real(), h->ymax = r.real(), h->zmax = r.real();
  h->hx = r.real(), h->hy = r.real(), h->hz = r.real();
  h->nx = (int)r.integer(), h->ny = (int)r.integer(), h->nz = (int)r.integer();
  r.raw();  // limp (logical)
  r.real(), r.real(), r.real();  // ximp, yimp, zimp
  const size_t N = (size_t)h->nx * h->ny * h->nz;
  den->resize(N);
  for (size_t k = 0; k < N; k++) (*den)[k] = r.real();
}

void read_impurity(const std::string &path, int *npar, std::vector<double> *rimp, std::vector<double> *vimp) {
  if (looks_binary(path, 4)) {
    FILE *f = fopen(path.c_str(), "rb");
    std::vector<char> rec;
    read_record(f, &rec);
    int32_t n = 0;
    memcpy(&n, rec.data(), 4);
    *npar = n;
    for (std::vector<double> *v : {rimp, vimp}) {
      if (!read_record(f, &rec) || rec.size() != 24 * (size_t)n) {
        fclose(f);
        throw std::runtime_error(path + ": particle record does not hold 3*N_par values");
      }
      v->resize(3 * (size_t)n);
      memcpy(v->data(), rec.data(), rec.size());
    }
    fclose(f);
    return;
  }
  const std::string s = slurp(path);
  ListReader r(s, after_comments(s));
  *npar = (int)r.integer();
  for (std::vector<double> *v : {rimp, vimp}) {
    v->resize(3 * (size_t)*npar);
    for (double &x : *v) x = r.real();
  }
}

std::string fmt_e(double v, int w, int d) {
  char b[64];
  snprintf(b, sizeof(b), "%*.*E", w, d, v);
  return b;
}

std::string fmt_f(double v, int w, int d) {
  char b[64];
  snprintf(b, sizeof(b), "%*.*f", w, d, v);
  return b;
}

static void cm_of(const GridHeader &h, const std::vector<std::complex<double>> &psi, double cm[3]) {
  double xn = 0, xc = 0, yc = 0, zc = 0;
  size_t t = 0;
  for (int iz = 0; iz < h.nz; iz++) {
    const double z = -h.zmax + iz * h.hz;
    for (int iy = 0; iy < h.ny; iy++) {
      const double y = -h.ymax + iy * h.hy;
      for (int ix = 0; ix < h.nx; ix++, t++) {
        const double sto = std::norm(psi[t]);
        xn += sto;
        xc += (-h.xmax + ix * h.hx) * sto;
        yc += y * sto;
        zc += z * sto;
      }
    }
  }
  cm[0] = xc / xn;
  cm[1] = yc / xn;
  cm[2] = zc / xn;
}

static void header(FILE *f, const PrintInfo &info, const double cm[3]) {
  fprintf(f, "#  Density after %15d iterations.\n", info.iter);
  fprintf(f, "#  Actual delatatps....:%s\n", fmt_e(info.paflv, 20, 10).c_str());
  fprintf(f, "#  Total evolution time(ps)...:%s\n", fmt_e(info.time, 20, 12).c_str());
  fprintf(f, "#  xcm,ycm,zcm:%s%s%s\n", fmt_e(cm[0], 16, 8).c_str(), fmt_e(cm[1], 16, 8).c_str(),
          fmt_e(cm[2], 16, 8).c_str());
  if (info.iprint == 1) fprintf(f, "#  Last printout of the run.\n");
  if (info.iprint == 2) fprintf(f, "#  Change of Paflov parameter.\n");
  if (info.iprint == 3) fprintf(f, "#  Backup copy.\n");
}

void write_psi(const std::string &path, const PrintInfo &info, const GridHeader &h,
               const std::vector<std::complex<double>> &psi) {
  FILE *f = fopen(path.c_str(), info.iprint < 0 ? "wb" : "w");
  if (!f) throw std::runtime_error("cannot write " + path);
  if (info.iprint < 0) {
    char rec[60];
    const double d[6] = {h.xmax, h.ymax, h.zmax, h.hx, h.hy, h.hz};
    const int32_t n[3] = {h.nx, h.ny, h.nz};
    memcpy(rec, d, 48);
    memcpy(rec + 48, n, 12);
    write_record(f, rec, 60);
    write_record(f, psi.data(), 16 * psi.size());
  } else {
    double cm[3];
    cm_of(h, psi, cm);
    header(f, info, cm);
    fprintf(f, " %.17E %.17E %.17E %.17E %.17E %.17E %d %d %d\n", h.xmax, h.ymax, h.zmax, h.hx, h.hy, h.hz, h.nx,
            h.ny, h.nz);
    for (const auto &c : psi) fprintf(f, " (%.17E,%.17E)\n", c.real(), c.imag());
  }
  fclose(f);
}

void write_impurity(const std::string &path, const PrintInfo &info, const GridHeader &h,
                    const std::vector<std::complex<double>> &psi, int npar, const std::vector<double> &rimp,
                    const std::vector<double> &vimp) {
  FILE *f = fopen(path.c_str(), info.iprint < 0 ? "wb" : "w");
  if (!f) throw std::runtime_error("cannot write " + path);
  if (info.iprint < 0) {
    const int32_t n = npar;
    write_record(f, &n, 4);
    write_record(f, rimp.data(), 8 * rimp.size());
    write_record(f, vimp.data(), 8 * vimp.size());
  } else {
    double cm[3];
    cm_of(h, psi, cm);
    header(f, info, cm);
    fprintf(f, " %d\n", npar);
    for (double x : rimp) fprintf(f, " %.17E\n", x);
    for (double x : vimp) fprintf(f, " %.17E\n", x);
  }
  fclose(f);
}

}  // namespace he4io
