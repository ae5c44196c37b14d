// he4io.hpp -- host-side input and output of the time-dependent run: the
// &input namelist (DFT4He3d.f90:147-187), readenc modes 0 and 2 (readenc.f90:78-114,
// with titols.f90's comment skipping) and printoutc (printoutc.f90:13-131),
// formatted (Fortran list-directed) and binary (Fortran unformatted
// sequential, 4-byte record markers).
#pragma once
#include <complex>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace he4io {

// A Fortran namelist group: names are lower-cased, values kept as written
// (strings without their quotes).
struct Namelist {
  std::string group;
  std::map<std::string, std::string> values;

  bool has(const std::string &k) const { return values.count(k) != 0; }
  std::string str(const std::string &k, const std::string &dflt) const;
  double real(const std::string &k, double dflt) const;  // accepts 1.5d-3
  long integer(const std::string &k, long dflt) const;
  bool logical(const std::string &k, bool dflt) const;   // .true. / T / .false. / F
};

// Parses the first namelist group named `group` from `text` (ignoring
// '!' comments outside strings).  Throws std::runtime_error on bad syntax.
Namelist parse_namelist(const std::string &text, const std::string &group);

// The grid header of a density / wave-function file.
struct GridHeader {
  double xmax = 0, ymax = 0, zmax = 0, hx = 0, hy = 0, hz = 0;
  int nx = 0, ny = 0, nz = 0;
};

// readenc mode 2: psi file (header line then psi(nx,ny,nz), complex) and
// impurity file (N_par, rimp(N_par,3), vimp(N_par,3)).  Lines whose first
// character is '#' before the data are skipped (titols).  Binary files
// (printoutc with iprint < 0) are recognised by their first record marker.
void read_psi(const std::string &path, GridHeader *hdr, std::vector<std::complex<double>> *psi);
void read_impurity(const std::string &path, int *npar, std::vector<double> *rimp, std::vector<double> *vimp);
// readenc mode 0 (readenc.f90:78-92): a real density file whose header line
// holds xmax,ymax,zmax,hx,hy,hz,nx,ny,nz,limp,ximp,yimp,zimp, then den(nx,ny,nz).
void read_density(const std::string &path, GridHeader *hdr, std::vector<double> *den);

// printoutc: iprint 1 (last printout), 2 (Paflov change) or 3 (backup)
// with the formatted header comments; iprint < 0 writes the binary form.
struct PrintInfo {
  double time = 0;      // total evolution time (ps)
  int iprint = 3;
  int iter = 0;
  double paflv = 0;     // written as "Actual delatatps"
};
void write_psi(const std::string &path, const PrintInfo &info, const GridHeader &hdr,
               const std::vector<std::complex<double>> &psi);
void write_impurity(const std::string &path, const PrintInfo &info, const GridHeader &hdr,
                    const std::vector<std::complex<double>> &psi, int npar, const std::vector<double> &rimp,
                    const std::vector<double> &vimp);

// Fortran-style real formatting: 1P Ew.d (one digit before the point).
std::string fmt_e(double v, int w, int d);
std::string fmt_f(double v, int w, int d);

}  // namespace he4io
