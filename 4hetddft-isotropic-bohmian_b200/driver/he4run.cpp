// he4run.cpp -- host driver of the time-dependent run: the C++ counterpart of
// the reference's Fortran main program around the time step
// (DFT4He3d.f90:147-243 input, :368 readenc, :621-660 first field and
// energy, :848-1045 the time loop, :1046 the last printout), calling the
// B200 library through include/he4_tddft.h.
//
//   he4run [--binary] < input.nml
//   he4run --roundtrip [--binary] psi_in imp_in psi_out imp_out
//   he4run --print-input < input.nml     (parse and read only)
//
// The &input namelist keeps the reference's names.  Additions for what the
// reference selects by code rather than by input: selec_gs = 'morse' with
// morse_d / morse_alpha / morse_re (the pair potential of the benchmark
// workloads), selec_gs = 'null', or vqfile = a tabulated Vq on the half
// spectrum; precision = 'fp64' | 'fp32conv'; device.  --binary writes the
// printoutc files in the iprint < 0 (unformatted) form; readenc reads either
// form.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/he4_tddft.h"
#include "he4io.hpp"

using he4io::fmt_e;
using he4io::fmt_f;

namespace {

constexpr double kKtops = 7.63822291;  // DFT4He3d.f90:104
constexpr double kPstoK = 1.0 / 7.63822291;

[[noreturn]] void die(const std::string &msg) {
  fprintf(stderr, "he4run: %s\n", msg.c_str());
  exit(1);
}

void check(int rc, const char *what) {
  if (rc != HE4_OK) die(std::string(what) + ": " + he4_last_error() + " (" + he4_strerror(rc) + ")");
}

std::string lower(std::string s) {
  for (char &c : s) c = (char)tolower((unsigned char)c);
  return s;
}

std::string three_digits(int n) {
  char b[16];
  snprintf(b, sizeof(b), "%03d", n);  // formats 8011-8013
  return b;
}

void print_energies(const he4_energies &e, double eold, int n4, double n4atoms) {
  // formats 7010 and 7015 (DFT4He3d.f90:1156-1170)
  printf("\n\n    ITERATIVE PROCEDURE \n\n");
  printf("    Total Energy (He).......... %s K +- %s K\n", fmt_f(e.etot4, 18, 6).c_str(),
         fmt_e(e.etot - eold, 12, 4).c_str());
  printf("    Energy per particle (He)... %s K\n\n", fmt_f(e.etot4 / n4, 18, 6).c_str());
  printf("    Kinetic Energy (He)........ %s K\n", fmt_f(e.ekin4, 18, 6).c_str());
  printf("    Lennard-Jones Energy (He).. %s K\n", fmt_f(e.elj4, 18, 6).c_str());
  printf("    Alpha_s term  energy (He).. %s K\n", fmt_f(e.ealphas, 18, 6).c_str());
  printf("    Solid energy (He) ......... %s K\n", fmt_f(e.esolid, 18, 6).c_str());
  printf("    Correlation Energy  (He)... %s K\n", fmt_f(e.ecor4, 18, 6).c_str());
  printf("    Impurity energy (X->He) ... %s K\n", fmt_f(e.eimpu, 18, 6).c_str());
  printf("    Kinetic energy (X) ........ %s K\n", fmt_f(e.ekinx, 18, 6).c_str());
  printf("    Kinetic Q-energy (X) ...... %s K\n", fmt_f(e.ekinqx, 18, 6).c_str());
  printf("    Interaction energy (X-He) . %s K\n", fmt_f(e.eHeX, 18, 6).c_str());
  printf("    Spin-Orbit energy (X) ..... %s K\n", fmt_f(0.0, 18, 6).c_str());
  printf("    TOTAL energy (He+X) ....... %s K\n \n", fmt_f(e.etot, 18, 6).c_str());
  (void)n4atoms;
}

void means_line(FILE *f, double time, double a, double b, double c) {
  fprintf(f, " %s%s%s%s\n", fmt_e(time, 15, 6).c_str(), fmt_e(a, 18, 10).c_str(), fmt_e(b, 18, 10).c_str(),
          fmt_e(c, 18, 10).c_str());
}

struct Run {
  he4_params p;
  he4io::GridHeader grid;
  std::vector<std::complex<double>> psi;
  std::vector<double> rimp, vimp, aimp;
  std::vector<double> vq;  // tabulated Vq (vqfile)
  std::vector<double> vr;  // sampled V(r) (vrfile)
  int npar = 0, n4 = 300, niter = 0, iter0 = 0, pener = 50, pcurr = 0, icurr = 0;
  bool lrk = false, binary = false;
  // spherical bubble radius of the pener block (DFT4He3d.f90:126-135,698-760)
  bool lbubble = false, lspherical = true;
  int nr = 501;
  std::string file_spherical_bubble;
  double deltat = 0, deltatps = 0, time0 = 0;
  std::string filedenin, fileimpin, filedenout, fileimpout, filerimp, filevimp, fileaimp;
  // readenc mode 0 start (DFT4He3d.f90:585-617): phase constraints, the box
  // the particles are drawn in, their common velocity (A/ps), the seed of
  // the draw (the reference's random_number is unseeded)
  int mode = 0;
  double xlamdax = 0, xlamday = 0, xlamdaz = 0;
  double xi = 1e99, xf = 1e99, yi = 1e99, yf = 1e99, zi = 1e99, zf = 1e99;
  double v0[3] = {0, 0, 0};
  unsigned long long seed = 1;
};

void load_input(Run &r, const std::string &text) {
  const he4io::Namelist nl = he4io::parse_namelist(text, "input");
  he4_params &p = r.p;
  he4_params_default(&p);
  p.nx = (int)nl.integer("nx", 64);
  p.ny = (int)nl.integer("ny", p.nx);
  p.nz = (int)nl.integer("nz", p.nx);
  p.xmax = nl.real("xmax", 0.0);
  p.ymax = nl.real("ymax", p.xmax);
  p.zmax = nl.real("zmax", p.xmax);
  p.npd = (int)nl.integer("npd", p.npd);
  p.icon = (int)nl.integer("icon", p.icon);
  const std::string core = lower(nl.str("core4", "OTC"));
  p.core4 = (core.rfind("otc", 0) == 0) ? HE4_CORE_OTC : HE4_CORE_OT;
  p.eps4 = nl.real("eps4", p.eps4);
  p.sigma4 = nl.real("sigma4", p.sigma4);
  p.cp4 = nl.real("cp4", p.cp4);
  p.cpp4 = nl.real("cpp4", p.cpp4);
  p.den4c = nl.real("den4c", p.den4c);
  p.alphas = nl.real("alphas", p.alphas);
  p.h2o2m4 = nl.real("h2o2m4", p.h2o2m4);
  p.nq = (int)nl.integer("nq", p.nq);
  p.mimpur = nl.real("mimpur", p.mimpur);
  p.n_par = (int)nl.integer("n_par", p.n_par);
  p.ironx = (int)nl.integer("ironx", p.ironx);
  p.lambdah = nl.real("lambdah", 0.0);
  p.tzmean = nl.real("tzmean", 0.0);
  p.tzsurf = nl.real("tzsurf", 1.0);
  p.device = (int)nl.integer("device", 0);
  const std::string prec = lower(nl.str("precision", "fp64"));
  if (prec == "fp64")
    p.precision = HE4_PREC_FP64;
  else if (prec == "fp32conv")
    p.precision = HE4_PREC_FP32CONV;
  else
    die("precision must be 'fp64' or 'fp32conv'");
  // impurity pair potential (Select_Pot, V_impur.f90:84-935)
  const std::string selec = lower(nl.str("selec_gs", "null"));
  p.r_cutoff = nl.real("r_cutoff_gs", p.r_cutoff);
  p.umax = nl.real("umax_gs", p.umax);
  if (nl.has("vqfile")) {
    p.pot_kind = HE4_POT_TABLE;
    std::ifstream f(nl.str("vqfile", ""));
    if (!f) die("cannot open vqfile");
    const size_t H = (size_t)(p.nx / 2 + 1) * p.ny * p.nz;
    r.vq.resize(H);
    for (size_t i = 0; i < H; i++)
      if (!(f >> r.vq[i])) die("vqfile holds fewer than (nx/2+1)*ny*nz values");
    p.vq_table = r.vq.data();
  } else if (nl.has("vrfile")) {
    // any Select_Pot entry sampled on a uniform r grid: lines "r V(r)" from
    // r_cutoff on; the library splines and Fourier-transforms it
    std::ifstream f(nl.str("vrfile", ""));
    if (!f) die("cannot open vrfile");
    std::vector<double> rs;
    double a, b;
    while (f >> a >> b) {
      rs.push_back(a);
      r.vr.push_back(b);
    }
    if (rs.size() < 4) die("vrfile holds fewer than 4 (r, V) pairs");
    const double dr = (rs.back() - rs.front()) / (double)(rs.size() - 1);
    for (size_t i = 1; i < rs.size(); i++)
      if (std::fabs(rs[i] - rs[i - 1] - dr) > 1e-6 * dr) die("vrfile r values are not uniformly spaced");
    p.pot_kind = HE4_POT_RTABLE;
    p.vr_table = r.vr.data();
    p.n_vr = (int32_t)r.vr.size();
    p.vr_r0 = rs.front();
    p.vr_dr = dr;
  } else if (selec == "morse") {
    p.pot_kind = HE4_POT_MORSE;
    p.morse_d = nl.real("morse_d", 10.0);
    p.morse_alpha = nl.real("morse_alpha", 1.2);
    p.morse_re = nl.real("morse_re", 5.5);
  } else if (selec == "null") {
    p.pot_kind = HE4_POT_NULL;
  } else if (selec == "he2s_fci") {
    p.pot_kind = HE4_POT_HE2S_FCI;  // evaluated by the library on the device
  } else {
    die("Select_Pot entry '" + selec +
        "' is not built into the library: sample its V(r) from r_cutoff_gs on into vrfile, or tabulate its Vq "
        "into vqfile");
  }
  r.n4 = (int)nl.integer("n4", 300);
  r.niter = (int)nl.integer("niter", 0);
  r.iter0 = (int)nl.integer("iter0", 0);
  r.pener = (int)nl.integer("pener", 50);
  r.pcurr = (int)nl.integer("pcurr", 0);
  r.icurr = (int)nl.integer("icurr", 0);
  r.time0 = nl.real("time0", 0.0);
  r.lrk = nl.logical("lrk", false);
  r.lbubble = nl.logical("lbubble_radius", false);
  r.lspherical = nl.logical("lspherical_bubble", true);
  r.nr = (int)nl.integer("nr", 501);
  r.file_spherical_bubble = nl.str("file_spherical_bubble", "spherical_bubble.out");
  // Delta t in K^-1 or ps (DFT4He3d.f90:229-243)
  r.deltat = nl.real("deltat", 0.0);
  r.deltatps = nl.real("deltatps", 0.0);
  if (r.deltat == 0.0) {
    if (r.deltatps == 0.0) die("You must specify either Deltat (in kelvin) or Deltatps (in picosecond)");
    r.deltat = r.deltatps / kKtops;
  } else if (r.deltatps == 0.0) {
    r.deltatps = r.deltat * kKtops;
  }
  r.mode = (int)nl.integer("mode", 0);
  if (r.mode != 0 && r.mode != 2) die("ERROR READEN: This mode is still not programmed");  // readenc.f90:116-121
  r.xlamdax = nl.real("xlamdax", 0.0);
  r.xlamday = nl.real("xlamday", 0.0);
  r.xlamdaz = nl.real("xlamdaz", 0.0);
  const double xlamda = nl.real("xlamda", 0.0);
  if (xlamda != 0.0) r.xlamdaz = xlamda * kKtops / (2.0 * p.h2o2m4);  // DFT4He3d.f90:579-582
  r.xi = nl.real("xi", 1e99), r.xf = nl.real("xf", 1e99);
  r.yi = nl.real("yi", 1e99), r.yf = nl.real("yf", 1e99);
  r.zi = nl.real("zi", 1e99), r.zf = nl.real("zf", 1e99);
  r.v0[0] = nl.real("v0x", 0.0), r.v0[1] = nl.real("v0y", 0.0), r.v0[2] = nl.real("v0z", 0.0);
  r.seed = (unsigned long long)nl.integer("seed", 1);
  // the reference asks for the particle box at every start (DFT4He3d.f90:188-196);
  // only the mode-0 draw uses it here
  if (r.mode == 0 && (r.xi > 1e10 || r.xf > 1e10 || r.yi > 1e10 || r.yf > 1e10 || r.zi > 1e10 || r.zf > 1e10))
    die("Has de definirme los limites de la impuerza... (xi, xf, yi, yf, zi, zf)");
  r.filedenin = nl.str("filedenin", "he4.input.density");
  r.fileimpin = nl.str("fileimpin", "X.input.wf");
  r.filedenout = nl.str("filedenout", "he4.output.density");
  r.fileimpout = nl.str("fileimpout", "X.output.wf");
  r.filerimp = nl.str("filerimp", "rimp.out");
  r.filevimp = nl.str("filevimp", "vimp.out");
  r.fileaimp = nl.str("fileaimp", "aimp.out");
}

void readenc_mode2(Run &r) {
  he4io::read_psi(r.filedenin, &r.grid, &r.psi);
  if (r.grid.nx != r.p.nx || r.grid.ny != r.p.ny || r.grid.nz != r.p.nz)
    die("the density file's grid does not match the namelist");
  int n = 0;
  he4io::read_impurity(r.fileimpin, &n, &r.rimp, &r.vimp);
  if (n != r.p.n_par) die("Readenc: --> N_par # N_Par0");  // readenc.f90:107-110
  r.npar = n;
  r.grid.hx = 2.0 * r.p.xmax / r.p.nx;
  r.grid.hy = 2.0 * r.p.ymax / r.p.ny;
  r.grid.hz = 2.0 * r.p.zmax / r.p.nz;
  r.grid.xmax = r.p.xmax, r.grid.ymax = r.p.ymax, r.grid.zmax = r.p.zmax;
}

// trilinear value of a grid field at a point, zero outside cells 1..n-1
// (interpola3denx with blend_103, sorteo.f90:49-83)
double trilinear(const std::vector<double> &f, const Run &r, const double xyz[3]) {
  const double lo[3] = {-r.p.xmax, -r.p.ymax, -r.p.zmax}, hh[3] = {r.grid.hx, r.grid.hy, r.grid.hz};
  const int n[3] = {r.p.nx, r.p.ny, r.p.nz};
  int ic[3];
  double w[3];
  for (int c = 0; c < 3; c++) {
    const double a = (xyz[c] - lo[c]) / hh[c] + 1.0;
    ic[c] = (int)a;
    w[c] = a - ic[c];
    if (ic[c] >= n[c] || ic[c] <= 0) return 0.0;
  }
  auto at = [&](int dx, int dy, int dz) {
    return f[((size_t)(ic[2] - 1 + dz) * r.p.ny + (ic[1] - 1 + dy)) * r.p.nx + (ic[0] - 1 + dx)];
  };
  double v = 0.0;
  for (int dz = 0; dz < 2; dz++)
    for (int dy = 0; dy < 2; dy++)
      for (int dx = 0; dx < 2; dx++)
        v += (dx ? w[0] : 1.0 - w[0]) * (dy ? w[1] : 1.0 - w[1]) * (dz ? w[2] : 1.0 - w[2]) * at(dx, dy, dz);
  return v;
}

// readenc mode 0 (readenc.f90:78-92) and the start it implies
// (DFT4He3d.f90:585-617): psi = sqrt(den) exp(i (lx x + ly y + lz z)); the
// test particles drawn by rejection from denx inside [xi,xf]x[yi,yf]x[zi,zf]
// (sorteo.f90:1-28, here from a seeded generator), all moving at v0
void readenc_mode0(Run &r) {
  std::vector<double> den, denx;
  he4io::GridHeader gx;
  he4io::read_density(r.filedenin, &r.grid, &den);
  he4io::read_density(r.fileimpin, &gx, &denx);
  if (r.grid.nx != r.p.nx || r.grid.ny != r.p.ny || r.grid.nz != r.p.nz || gx.nx != r.p.nx || gx.ny != r.p.ny ||
      gx.nz != r.p.nz)
    die("the density files' grid does not match the namelist");
  r.grid.hx = 2.0 * r.p.xmax / r.p.nx;
  r.grid.hy = 2.0 * r.p.ymax / r.p.ny;
  r.grid.hz = 2.0 * r.p.zmax / r.p.nz;
  r.grid.xmax = r.p.xmax, r.grid.ymax = r.p.ymax, r.grid.zmax = r.p.zmax;
  r.psi.resize(den.size());
  for (int iz = 0; iz < r.p.nz; iz++)
    for (int iy = 0; iy < r.p.ny; iy++)
      for (int ix = 0; ix < r.p.nx; ix++) {
        const double x = -r.p.xmax + r.grid.hx * ix, y = -r.p.ymax + r.grid.hy * iy, z = -r.p.zmax + r.grid.hz * iz;
        const double aux = x * r.xlamdax + y * r.xlamday + z * r.xlamdaz;
        const size_t t = ((size_t)iz * r.p.ny + iy) * r.p.nx + ix;
        r.psi[t] = std::sqrt(den[t]) * std::complex<double>(std::cos(aux), std::sin(aux));
      }
  double dmax = 0.0;
  for (double v : denx) dmax = std::max(dmax, v);
  if (!(dmax > 0.0)) die("sorteo: the impurity density is zero everywhere");
  const int np = r.p.n_par;
  r.npar = np;
  r.rimp.assign(3 * (size_t)np, 0.0);
  r.vimp.assign(3 * (size_t)np, 0.0);
  std::mt19937_64 gen(r.seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  const double lo[3] = {r.xi, r.yi, r.zi}, hi[3] = {r.xf, r.yf, r.zf};
  for (int i = 0; i < np; i++) {
    double xyz[3];
    for (long tries = 0;; tries++) {
      if (tries > 100000000L) die("sorteo: no particle accepted in 1e8 draws (box outside denx?)");
      for (int c = 0; c < 3; c++) xyz[c] = u(gen) * (hi[c] - lo[c]) + lo[c];
      const double dum = u(gen) * dmax;
      if (dum < trilinear(denx, r, xyz)) break;
    }
    for (int c = 0; c < 3; c++) {
      r.rimp[(size_t)c * np + i] = xyz[c];
      r.vimp[(size_t)c * np + i] = r.v0[c] * kKtops;  // A/ps -> A*K
    }
  }
  // density.000.dat / densityx.000.dat of the start (DFT4He3d.f90:611-617)
  he4io::PrintInfo info;
  info.time = 0.0;
  info.iprint = r.binary ? -3 : 3;
  info.iter = 0;
  info.paflv = r.deltatps;
  he4io::write_psi("density.000.dat", info, r.grid, r.psi);
  he4io::write_impurity("densityx.000.dat", info, r.grid, r.psi, r.npar, r.rimp, r.vimp);
}

void printoutc(he4_handle *h, Run &r, double time, int iprint, const std::string &f, const std::string &f1,
               int iter) {
  r.aimp.resize(r.rimp.size());
  check(he4_get_state(h, reinterpret_cast<double *>(r.psi.data()), r.rimp.data(), r.vimp.data(), r.aimp.data()),
        "he4_get_state");
  he4io::PrintInfo info;
  info.time = time;
  info.iprint = r.binary ? -std::abs(iprint) : iprint;
  info.iter = iter;
  info.paflv = r.deltatps;
  he4io::write_psi(f, info, r.grid, r.psi);
  he4io::write_impurity(f1, info, r.grid, r.psi, r.npar, r.rimp, r.vimp);
}

// printoutc backups every pcurr steps (DFT4He3d.f90:992-1009) without
// stopping the time loop: the library snapshots the state and copies it to
// pinned host memory while the next step runs; the files are then written
// by a writer thread while the loop goes on.
struct Backup {
  bool pending = false;  // snapshot in flight, not yet collected
  int iter = 0;
  double time = 0.0;
  std::string f, f1;
  std::thread writer;
};

void backup_begin(he4_handle *h, Backup &b, double time, int iter, const std::string &f, const std::string &f1) {
  if (b.writer.joinable()) b.writer.join();  // the pinned copy is reused
  check(he4_snapshot_begin(h), "he4_snapshot_begin");
  b.pending = true;
  b.iter = iter;
  b.time = time;
  b.f = f;
  b.f1 = f1;
}

void backup_collect(he4_handle *h, Run &r, Backup &b) {
  if (!b.pending) return;
  const double *psi = nullptr, *rimp = nullptr, *vimp = nullptr;
  check(he4_snapshot_wait(h, &psi, &rimp, &vimp, nullptr), "he4_snapshot_wait");
  b.pending = false;
  he4io::PrintInfo info;
  info.time = b.time;
  info.iprint = r.binary ? -3 : 3;
  info.iter = b.iter;
  info.paflv = r.deltatps;
  const size_t N = (size_t)r.p.nx * r.p.ny * r.p.nz, P3 = 3 * (size_t)r.npar;
  const he4io::GridHeader grid = r.grid;
  const int npar = r.npar;
  const std::string f = b.f, f1 = b.f1;
  b.writer = std::thread([=]() {
    std::vector<std::complex<double>> ps(reinterpret_cast<const std::complex<double> *>(psi),
                                         reinterpret_cast<const std::complex<double> *>(psi) + N);
    std::vector<double> ri(rimp, rimp + P3), vi(vimp, vimp + P3);
    he4io::write_psi(f, info, grid, ps);
    he4io::write_impurity(f1, info, grid, ps, npar, ri, vi);
  });
}

void denx_cuts(he4_handle *h, const Run &r, const double means[9]) {
  const size_t N = (size_t)r.p.nx * r.p.ny * r.p.nz;
  std::vector<double> denx(N);
  check(he4_get_field(h, HE4_F_DENX, denx.data()), "he4_get_field");
  // NGP cell of the mean position (DFT4He3d.f90:894-896), clamped to the grid
  auto cell = [](double a, double x0, double hh, int n) {
    int i = (int)(1.5 + (a + x0) / hh) - 1;
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
  };
  const int ipx = cell(means[0], r.p.xmax, r.grid.hx, r.p.nx);
  const int ipy = cell(means[1], r.p.ymax, r.grid.hy, r.p.ny);
  const int ipz = cell(means[2], r.p.zmax, r.grid.hz, r.p.nz);
  auto at = [&](int ix, int iy, int iz) { return denx[((size_t)iz * r.p.ny + iy) * r.p.nx + ix]; };
  FILE *f = fopen("denx-x.dat", "w");
  for (int ix = 0; ix < r.p.nx; ix++)
    fprintf(f, "%s%s\n", fmt_e(-r.p.xmax + ix * r.grid.hx, 15, 6).c_str(), fmt_e(at(ix, ipy, ipz), 15, 6).c_str());
  fclose(f);
  f = fopen("denx-y.dat", "w");
  for (int iy = 0; iy < r.p.ny; iy++)
    fprintf(f, "%s%s\n", fmt_e(-r.p.ymax + iy * r.grid.hy, 15, 6).c_str(), fmt_e(at(ipx, iy, ipz), 15, 6).c_str());
  fclose(f);
  f = fopen("denx-z.dat", "w");
  for (int iz = 0; iz < r.p.nz; iz++)
    fprintf(f, "%s%s\n", fmt_e(-r.p.zmax + iz * r.grid.hz, 15, 6).c_str(), fmt_e(at(ipx, ipy, iz), 15, 6).c_str());
  fclose(f);
}

// Lbubble_radius block (DFT4He3d.f90:929-986): the impurity mean-square
// radii, then with Lspherical_bubble the spherical bubble radius, written
// to file_spherical_bubble when both searches succeed.  The axial radii of
// bubble_radius.f90 are not computed.
void bubble_block(he4_handle *h, const Run &r, FILE *f62, double time) {
  if (!r.lbubble) return;
  double rb = 0.0, xms[3];
  int32_t found[2] = {0, 0}, ir = 0;
  check(he4_bubble_radius(h, r.nr, &rb, found, &ir, xms, nullptr, nullptr), "he4_bubble_radius");
  printf(" Impurity mean square radius:(X),(Y),(Z): %s%s%s\n", fmt_e(xms[0], 15, 6).c_str(),
         fmt_e(xms[1], 15, 6).c_str(), fmt_e(xms[2], 15, 6).c_str());
  if (r.lspherical && found[0] && found[1]) {
    printf("Spherical bubble radius........:%s\n", fmt_e(rb, 15, 6).c_str());
    fprintf(f62, "%s%s\n", fmt_e(time, 15, 6).c_str(), fmt_e(rb, 18, 10).c_str());
    fflush(f62);
  }
}

int roundtrip(int argc, char **argv, bool binary) {
  if (argc < 4) die("--roundtrip needs psi_in imp_in psi_out imp_out");
  he4io::GridHeader g;
  std::vector<std::complex<double>> psi;
  std::vector<double> rimp, vimp;
  int n = 0;
  he4io::read_psi(argv[0], &g, &psi);
  he4io::read_impurity(argv[1], &n, &rimp, &vimp);
  he4io::PrintInfo info;
  info.iprint = binary ? -3 : 3;
  he4io::write_psi(argv[2], info, g, psi);
  he4io::write_impurity(argv[3], info, g, psi, n, rimp, vimp);
  printf("%d %d %d %d\n", g.nx, g.ny, g.nz, n);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  Run r;
  int a = 1;
  bool rt = false, show = false;
  for (; a < argc && argv[a][0] == '-'; a++) {
    if (!strcmp(argv[a], "--binary"))
      r.binary = true;
    else if (!strcmp(argv[a], "--roundtrip"))
      rt = true;
    else if (!strcmp(argv[a], "--print-input"))
      show = true;
    else
      die(std::string("unknown option ") + argv[a]);
  }
  try {
    if (rt) return roundtrip(argc - a, argv + a, r.binary);
    std::stringstream ss;
    ss << std::cin.rdbuf();
    load_input(r, ss.str());
    if (r.mode == 0)
      readenc_mode0(r);
    else
      readenc_mode2(r);
  } catch (const std::exception &e) {
    die(e.what());
  }
  if (show) {  // the parsed input, without touching a GPU
    const he4_params &p = r.p;
    printf("nx=%d ny=%d nz=%d xmax=%.17g ymax=%.17g zmax=%.17g npd=%d icon=%d core4=%d\n", p.nx, p.ny, p.nz,
           p.xmax, p.ymax, p.zmax, p.npd, p.icon, p.core4);
    printf("n_par=%d pot_kind=%d r_cutoff=%.17g umax=%.17g precision=%d\n", p.n_par, p.pot_kind, p.r_cutoff, p.umax,
           p.precision);
    printf("deltat=%.17g deltatps=%.17g niter=%d pener=%d pcurr=%d\n", r.deltat, r.deltatps, r.niter, r.pener,
           r.pcurr);
    printf("n_vr=%d vr_r0=%.17g vr_dr=%.17g lbubble=%d lspherical=%d nr=%d\n", p.n_vr, p.vr_r0, p.vr_dr,
           (int)r.lbubble, (int)r.lspherical, r.nr);
    double s = 0;
    for (const auto &c : r.psi) s += std::norm(c);
    printf("psi_norm2=%.17g rimp0=%.17g vimp_last=%.17g\n", s, r.rimp[0], r.vimp.back());
    return 0;
  }
  he4_handle *h = nullptr;
  check(he4_create(&r.p, &h), "he4_create");
  check(he4_set_state(h, reinterpret_cast<const double *>(r.psi.data()), r.rimp.data(), r.vimp.data()),
        "he4_set_state");
  FILE *f81 = fopen(r.filerimp.c_str(), "w"), *f82 = fopen(r.filevimp.c_str(), "w"),
       *f83 = fopen(r.fileaimp.c_str(), "w");
  if (!f81 || !f82 || !f83) die("cannot open the trajectory files");
  FILE *f62 = nullptr;
  if (r.lbubble && r.lspherical) {
    f62 = fopen(r.file_spherical_bubble.c_str(), "w");
    if (!f62) die("cannot open file_spherical_bubble");
  }
  // first field and energy (DFT4He3d.f90:630-660)
  check(he4_field(h), "he4_field");
  double diag[4];
  check(he4_diagnostics(h, r.n4, diag), "he4_diagnostics");
  std::vector<double> aimp(r.rimp.size());
  check(he4_get_state(h, nullptr, nullptr, nullptr, aimp.data()), "he4_get_state");
  double m0[9] = {0};
  for (int c = 0; c < 3; c++)
    for (int i = 0; i < r.npar; i++) {
      m0[c] += r.rimp[(size_t)c * r.npar + i] / r.npar;
      m0[3 + c] += r.vimp[(size_t)c * r.npar + i] / r.npar;
      m0[6 + c] += aimp[(size_t)c * r.npar + i] / r.npar;
    }
  fprintf(f81, "# Tiempo(ps), x(AA), y(AA), z(AA)\n");
  means_line(f81, r.time0, m0[0], m0[1], m0[2]);
  fprintf(f82, "# Tiempo(ps), Vx(AA/ps), Vy(AA/ps), Vz(AA/ps)\n");
  means_line(f82, r.time0, m0[3] * kPstoK, m0[4] * kPstoK, m0[5] * kPstoK);
  fprintf(f83, "# Tiempo(ps), Ax(AA/ps**2), Ay(AA/ps**2), Az(AA/ps**2)\n");
  means_line(f83, r.time0, m0[6] * kPstoK * kPstoK, m0[7] * kPstoK * kPstoK, m0[8] * kPstoK * kPstoK);
  he4_energies e;
  check(he4_energy(h, &e), "he4_energy");
  printf("Number of He4 atoms%s\n", fmt_e(diag[0], 15, 6).c_str());
  bubble_block(h, r, f62, r.time0);
  double eold = e.etot;
  // the time loop (DFT4He3d.f90:848-1045)
  const int first = r.iter0 + 1;
  Backup bk;
  int iter = first;
  double time = r.time0;
  for (; iter <= r.niter; iter++) {
    double err[3] = {0, 0, 0}, means[9];
    if (iter <= first + 2 || r.lrk) {
      check(he4_step_rk(h, r.deltat, means), "he4_step_rk");
    } else {
      check(he4_step_pc(h, r.deltat, err, means), "he4_step_pc");
      printf("Err(He, rimp, vimp)..;%s%s%s\n", fmt_e(err[0], 15, 6).c_str(), fmt_e(err[1], 15, 6).c_str(),
             fmt_e(err[2], 15, 6).c_str());
    }
    time = r.time0 + (iter - first + 1) * r.deltatps;
    means_line(f81, time, means[0], means[1], means[2]);
    means_line(f82, time, means[3] * kPstoK, means[4] * kPstoK, means[5] * kPstoK);
    means_line(f83, time, means[6] * kPstoK * kPstoK, means[7] * kPstoK * kPstoK, means[8] * kPstoK * kPstoK);
    if (r.pener > 0 && iter % r.pener == 0) {
      check(he4_energy(h, &e), "he4_energy");
      check(he4_diagnostics(h, r.n4, diag), "he4_diagnostics");
      printf("Iteration........:%15d\n", iter);
      printf("Number of He4 atoms%s\n", fmt_e(diag[0], 15, 6).c_str());
      print_energies(e, eold, r.n4, diag[0]);
      eold = e.etot;
      printf("C.M. He..:%s%s%s\n", fmt_e(diag[1], 15, 6).c_str(), fmt_e(diag[2], 15, 6).c_str(),
             fmt_e(diag[3], 15, 6).c_str());
      printf("C.M. X..:%s%s%s\n", fmt_e(means[0], 15, 6).c_str(), fmt_e(means[1], 15, 6).c_str(),
             fmt_e(means[2], 15, 6).c_str());
      printf("C.M. V..:%s%s%s\n", fmt_e(means[3], 15, 6).c_str(), fmt_e(means[4], 15, 6).c_str(),
             fmt_e(means[5], 15, 6).c_str());
      denx_cuts(h, r, means);
      bubble_block(h, r, f62, time);
      fflush(stdout);
    }
    // the snapshot taken one step ago has reached host memory: write it
    if (bk.pending && iter > bk.iter) backup_collect(h, r, bk);
    if (r.pcurr > 0 && iter % r.pcurr == 0) {
      const int ncurr = (iter - first + 1) / r.pcurr + r.icurr;
      const std::string tag = three_digits(ncurr);
      backup_begin(h, bk, time, iter, "density." + tag + ".dat", "densityx." + tag + ".dat");
    }
  }
  backup_collect(h, r, bk);
  if (bk.writer.joinable()) bk.writer.join();
  fclose(f81);
  fclose(f82);
  fclose(f83);
  if (f62) fclose(f62);
  printoutc(h, r, time, 1, r.filedenout, r.fileimpout, iter);
  he4_destroy(h);
  return 0;
}
