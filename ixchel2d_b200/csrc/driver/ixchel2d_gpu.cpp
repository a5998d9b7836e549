// ixchel2d_gpu.cpp -- PROGRAM IXCHEL2D (source/main.f90) on libixb.
//
// Reads a case folder exactly as the reference does and writes the same
// files, with the time loop on the GPU through the C ABI of include/ixb.h:
//
// * parametros.dat: the 23 list-directed records of main.f90:164-189
//   (adimen, Ra, Pr, Ri_1, dt, paq_itera, itermax, rel_pres, rel_vel,
//   rel_ener, conv_u, conv_t, conv_p, conv_resi, conv_paso, iter_ecuaci_max,
//   iter_simple_max, entrada_u, entrada_v, entrada_tp, flujo_ini, tempe_ini,
//   postprocesar), non-dimensionalised as main.f90:215-244;
// * n<nj>m<mi>R<Re>/info_entrada.out (postprocesa_parametros,
//   mod_postproceso.f90:26-90); the folder must exist, as for the reference;
// * the three mesh/state files named by entrada_u/v/tp
//   (lectura_mallas_escalonadas, mod_malla.f90:137-162);
// * the initial conditions of condicion_inicial_flujo / _tempe
//   (mod_ec_momento.f90:59-89, mod_ec_energia.f90:46-80) and main.f90:302-317;
// * cond_frontera{u,v,t}.dat (ini_frontera_uv / _t, mod_ec_momento.f90:100-134,
//   mod_ec_energia.f90:98-110);
// * the time loop of main.f90:350-1378: itermax/paq_itera packages of
//   paq_itera time steps (ixb_step = the ALGORITMO_SIMPLE loop plus the roll),
//   "ITERACION:" every 500 steps, the record (time, Nu0, -Nu1, T_med,
//   T_int, S_int) in form26 appended to nuss_sim_n<nj>m<mi>_R<Re>.dat every
//   1000 steps, and after every package the summary lines and, when
//   postprocesar is true, out_n<nj>m<mi>_R<Re>{u,v,p}.dat (form24/form25),
//   out_..{u,v,p}.bin (postproceso_bin, mod_postproceso.f90:310-365) and the
//   big-endian VTK file n<nj>m<mi>R<Re>/t_<mcdud>.vtk (postproceso_vtk,
//   :225-300).  The package's state leaves the device through
//   ixb_download_state_async (a snapshot copied to pinned host buffers on the
//   library's download stream), and a writer thread formats and writes these
//   files while the next package runs on the GPU.
//
// mi and nj are compile-time parameters of the reference (mod_malla.f90:15);
// here they are taken from the record counts of the mesh files, or from
// --mi/--nj.  Differences from the reference, all where its behaviour is
// undefined or a crash: temp_int, entropia_int, lambda_ent and a_ent are
// never set by the reference (uninitialised locals) and are written as 0;
// Res_T and Res_v are never computed there (zero module arrays) and are
// printed as 0; the per-iteration 'SIMPLE' lines of unit 102 (fort.102) are
// not written; paq_itera < 10 divides by zero in the reference's VTK name
// (main.f90:1283-1284) and gives the tenths digit 0 here; a NaN or Inf in a
// convergence norm stops the run (status 3) where the reference iterates on.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/ixb.h"
#include "../ixb_listdir.h"

namespace {

using ixb::fmt_d23_15;

// parametros.dat after the READs of main.f90:164-189
struct Parametros {
  std::string adimen;  // character(len=7)
  double Ra = 0, Pr = 0, Ri_1 = 0, dt = 0;
  int paq_itera = 0, itermax = 0;
  double rel_pres = 0, rel_vel = 0, rel_ener = 0;
  double conv_u = 0, conv_t = 0, conv_p = 0, conv_resi = 0, conv_paso = 0;
  int iter_ecuaci_max = 0, iter_simple_max = 0;
  std::string entrada_u, entrada_v, entrada_tp;  // character(len=28)
  std::string flujo_ini, tempe_ini;              // character(len=8)
  int postprocesar = 0;
};

struct Options {
  std::string dir;
  int mi = 0, nj = 0;
  int prec = IXB_PREC_FP64;
  int solver = IXB_SOLVER_HYBRID;
  int cuerpo = -1;  // definir_cuerpo option; -1 = 'sincu', the reference's choice (main.f90:327)
  bool autotune = true, check = false, mkdir = false, quiet = false;
};

[[noreturn]] void die(int code, const std::string& msg) {
  std::fprintf(stderr, "ixchel2d_gpu: %s\n", msg.c_str());
  std::exit(code);
}

std::string rtrim(std::string s) {
  while (!s.empty() && s.back() == ' ') s.pop_back();
  return s;
}

bool read_parametros(const char* path, Parametros* P, std::string* err) {
  ixb::ListReader rd(path);
  if (!rd.ok()) { *err = std::string("cannot open ") + path; return false; }
  std::vector<std::string> it;
  int rec = 0;
  auto next = [&](const char* name) -> const std::string& {
    ++rec;
    if (!rd.read(it, 1)) {
      *err = std::string(path) + ": end of file at record " + std::to_string(rec) + " (" + name + ")";
      static const std::string none;
      return none;
    }
    return it[0];
  };
  auto real = [&](const char* name, double* v) {
    if (!err->empty()) return;
    const std::string& t = next(name);
    if (err->empty() && !ixb::parse_real(t, v))
      *err = std::string(path) + ": record " + std::to_string(rec) + " (" + name + "): not a real: '" + t + "'";
  };
  auto integer = [&](const char* name, int* v) {
    if (!err->empty()) return;
    const std::string& t = next(name);
    if (err->empty() && !ixb::parse_int(t, v))
      *err = std::string(path) + ": record " + std::to_string(rec) + " (" + name + "): not an integer: '" + t + "'";
  };
  auto chars = [&](const char* name, size_t len, std::string* v) {
    if (!err->empty()) return;
    const std::string& t = next(name);
    if (err->empty()) *v = rtrim(ixb::fortran_char(t, len));
  };
  auto logical = [&](const char* name, int* v) {
    if (!err->empty()) return;
    const std::string& t = next(name);
    if (err->empty() && !ixb::parse_logical(t, v))
      *err = std::string(path) + ": record " + std::to_string(rec) + " (" + name + "): not a logical: '" + t + "'";
  };
  err->clear();
  chars("adimen", 7, &P->adimen);
  real("Ra", &P->Ra);
  real("Pr", &P->Pr);
  real("Ri_1", &P->Ri_1);
  real("dt", &P->dt);
  integer("paq_itera", &P->paq_itera);
  integer("itermax", &P->itermax);
  real("rel_pres", &P->rel_pres);
  real("rel_vel", &P->rel_vel);
  real("rel_ener", &P->rel_ener);
  real("conv_u", &P->conv_u);
  real("conv_t", &P->conv_t);
  real("conv_p", &P->conv_p);
  real("conv_resi", &P->conv_resi);
  real("conv_paso", &P->conv_paso);
  integer("iter_ecuaci_max", &P->iter_ecuaci_max);
  integer("iter_simple_max", &P->iter_simple_max);
  chars("entrada_u", 28, &P->entrada_u);
  chars("entrada_v", 28, &P->entrada_v);
  chars("entrada_tp", 28, &P->entrada_tp);
  chars("flujo_ini", 8, &P->flujo_ini);
  chars("tempe_ini", 8, &P->tempe_ini);
  logical("postprocesar", &P->postprocesar);
  return err->empty();
}

// A one-digit I1 edit of an integer: '*' when it does not fit.
char digit(int d) { return (d >= 0 && d <= 9) ? (char)('0' + d) : '*'; }

// entero_caracter (mod_postproceso.f90:375-401): five I1 digits, ten
// thousands first; trimmed of the trailing blank of its character(6) result.
std::string entero_caracter(int e) {
  const int dmi = e / 10000;
  const int mil = (e - dmi * 10000) / 1000;
  const int cen = (e - dmi * 10000 - mil * 1000) / 100;
  const int dec = (e - dmi * 10000 - mil * 1000 - cen * 100) / 10;
  const int uni = e - dmi * 10000 - mil * 1000 - cen * 100 - dec * 10;
  return std::string{digit(dmi), digit(mil), digit(cen), digit(dec), digit(uni)};
}

// List-directed output of a REAL(8) (gfortran's form): 17 significant
// digits, fixed notation for 0.1 <= |x| < 1e17, otherwise E with a 3-digit
// exponent; 26 columns.
std::string fg(double x) {
  char b[64];
  const double a = std::fabs(x);
  std::string s;
  if (x == 0.0) {
    s = "0.0000000000000000     ";
  } else if (std::isfinite(x) && a >= 0.1 && a < 1e17) {
    const int e = (int)std::floor(std::log10(a)) + 1;
    std::snprintf(b, sizeof b, "%.*f", std::max(0, 17 - e), x);
    s = std::string(b) + "     ";
  } else if (std::isfinite(x)) {
    std::snprintf(b, sizeof b, "%.16E", x);
    std::string m(b);
    const size_t k = m.find('E');
    const int ex = std::atoi(m.c_str() + k + 1);
    std::snprintf(b, sizeof b, "E%c%03d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    s = m.substr(0, k) + b;
  } else {
    s = std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity");
  }
  if (s.size() < 26) s.insert(0, 26 - s.size(), ' ');
  return s;
}

std::string fi(int64_t v) {
  char b[32];
  std::snprintf(b, sizeof b, "%12lld", (long long)v);
  return b;
}

// Records after the list-directed header line: one per node in the D23.15 files.
long count_records(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return -1;
  long n = 0;
  bool first = true, blank = true;
  int ch;
  while ((ch = std::fgetc(f)) != EOF) {
    if (ch == '\n') {
      if (!first && !blank) ++n;
      first = false;
      blank = true;
    } else if (ch != ' ' && ch != '\t' && ch != '\r') {
      blank = false;
    }
  }
  if (!first && !blank) ++n;
  std::fclose(f);
  return n;
}

void parse_args(int argc, char** argv, Options* o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&]() -> std::string {
      if (i + 1 >= argc) die(2, "missing value after " + a);
      return argv[++i];
    };
    if (a == "--mi") o->mi = std::atoi(val().c_str());
    else if (a == "--nj") o->nj = std::atoi(val().c_str());
    else if (a == "--prec") {
      const std::string v = val();
      if (v == "fp64") o->prec = IXB_PREC_FP64;
      else if (v == "refined") o->prec = IXB_PREC_FP32_REFINED;
      else die(2, "--prec takes fp64 or refined");
    } else if (a == "--solver") {
      const std::string v = val();
      if (v == "hybrid") o->solver = IXB_SOLVER_HYBRID;
      else if (v == "exact") o->solver = IXB_SOLVER_EXACT;
      else die(2, "--solver takes hybrid or exact");
    } else if (a == "--cuerpo") {
      const std::string v = val();
      if (v == "sincu") o->cuerpo = -1;
      else if (v == "trian") o->cuerpo = IXB_BODY_TRIAN;
      else if (v == "cuadr") o->cuerpo = IXB_BODY_CUADR;
      else if (v == "chime") o->cuerpo = IXB_BODY_CHIME;
      else die(2, "--cuerpo takes sincu, trian, cuadr or chime");
    } else if (a == "--autotune") o->autotune = true;
    else if (a == "--no-autotune") o->autotune = false;
    else if (a == "--check") o->check = true;
    else if (a == "--mkdir") o->mkdir = true;
    else if (a == "--quiet") o->quiet = true;
    else if (a == "-h" || a == "--help") {
      std::printf(
          "usage: ixchel2d_gpu [CASE_DIR] [--mi M --nj N] [--prec fp64|refined] [--solver hybrid|exact]\n"
          "                    [--cuerpo sincu|trian|cuadr|chime] [--no-autotune] [--mkdir] [--check] [--quiet]\n"
          "Runs the Ixchel2D case in CASE_DIR (default: the current folder) on the GPU.\n"
          "--check reads every input, prints what it found and exits without using the GPU.\n"
          "The launch shapes of the line sweeps are autotuned on the initial state (--no-autotune: defaults).\n");
      std::exit(0);
    } else if (!a.empty() && a[0] == '-') die(2, "unknown option " + a);
    else o->dir = a;
  }
}

void ck(int st, const char* what) {
  if (st != IXB_OK) die(3, std::string(what) + ": " + ixb_strerror(st));
}

void put_be_float(std::string* out, double x) {
  const float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const char b[4] = {(char)(u >> 24), (char)(u >> 16), (char)(u >> 8), (char)u};
  out->append(b, 4);
}

bool write_file(const std::string& path, const std::string& bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
  return std::fclose(f) == 0 && ok;
}

template <class... A>
void put_doubles(std::string* out, A... x) {
  const double v[] = {x...};
  out->append(reinterpret_cast<const char*>(v), sizeof v);
}

}  // namespace

int main(int argc, char** argv) {
  Options opt;
  parse_args(argc, argv, &opt);
  if (!opt.dir.empty() && chdir(opt.dir.c_str()) != 0) die(2, "cannot enter " + opt.dir);
  const bool say = !opt.quiet;

  if (say) {
    std::printf(" ------------------------------------------\n  \n                  IXCHEL2D\n  \n"
                " ------------------------------------------\n Inicia lectura de archivo de par'ametros\n");
  }
  Parametros P;
  std::string err;
  if (!read_parametros("parametros.dat", &P, &err)) die(2, err);
  if (say) std::printf(" Finaliza lectura de archivo de par'ametros\n ------------------------------------------\n");

  // non-dimensionalisation, main.f90:213-244
  double gamma_momen, gamma_energ, Ri, Riy;
  std::string Rec;
  if (P.adimen == "natural") {
    gamma_momen = std::sqrt(P.Pr / P.Ra);
    gamma_energ = std::sqrt(1.0 / (P.Pr * P.Ra));
    Ri = 0.0;
    Riy = -1.0;
    Rec = entero_caracter((int)std::ceil(std::sqrt(P.Ra)));
  } else if (P.adimen == "mixta") {
    gamma_momen = 1.0 / P.Ra;
    gamma_energ = 1.0 / (P.Ra * P.Pr);
    Ri = 0.0;
    Riy = P.Ri_1;
    Rec = entero_caracter((int)std::ceil(P.Ra));
  } else {
    die(2, "parametros.dat: adimen must be 'natural' or 'mixta', not '" + P.adimen + "'");
  }
  if (P.paq_itera <= 0) die(2, "parametros.dat: paq_itera must be positive");

  // grid sizes from the record counts: u (mi, nj+1), v (mi+1, nj), p (mi+1, nj+1)
  int mi = opt.mi, nj = opt.nj;
  {
    const long nu = count_records(P.entrada_u), nv = count_records(P.entrada_v), np = count_records(P.entrada_tp);
    if (nu < 0) die(2, "cannot open " + P.entrada_u);
    if (nv < 0) die(2, "cannot open " + P.entrada_v);
    if (np < 0) die(2, "cannot open " + P.entrada_tp);
    if (mi == 0 && nj == 0) {
      const long nj1 = np - nu;
      if (nj1 < 3 || nu % nj1 != 0) die(2, "cannot infer mi, nj from the mesh files (give --mi and --nj)");
      nj = (int)(nj1 - 1);
      mi = (int)(nu / nj1);
    }
    if (mi < 2 || nj < 2) die(2, "mi and nj must both be given and at least 2");
    if (nu != (long)mi * (nj + 1) || nv != (long)(mi + 1) * nj || np != (long)(mi + 1) * (nj + 1))
      die(2, "the mesh files do not hold an (mi, nj) = (" + std::to_string(mi) + ", " + std::to_string(nj) +
                 ") staggered mesh");
  }
  const std::string mic = entero_caracter(mi), njc = entero_caracter(nj);
  const std::string folder = "n" + njc + "m" + mic + "R" + Rec;
  const std::string tag = "n" + njc + "m" + mic + "_R" + Rec;

  // mesh, state and boundary conditions
  std::vector<double> xu(mi), yv(nj), xp(mi + 1), yp(nj + 1);
  const size_t NU = (size_t)mi * (nj + 1), NV = (size_t)(mi + 1) * nj, NP = (size_t)(mi + 1) * (nj + 1);
  std::vector<double> u(NU), v(NV), p(NP), T(NP), u_ant(NU), v_ant(NV), T_ant(NP);
  int placa_min = 0, placa_max = 0, itera_inicial = 0;
  double ao = 0.0;
  ixb_bc_side bcu[4], bcv[4], bct[4];

  if (opt.mkdir) ::mkdir(folder.c_str(), 0755);
  {
    // postprocesa_parametros: fails, as the reference does, when the folder is missing
    const std::string info = folder + "/info_entrada.out";
    FILE* f = std::fopen(info.c_str(), "w");
    if (!f) die(2, "cannot open " + info + " (create the folder " + folder + "/, or pass --mkdir)");
    auto line = [&](const char* label, const std::string& val) { std::fprintf(f, " %s%s\n", label, val.c_str()); };
    auto pad = [](const std::string& s, size_t n) { return s + std::string(n > s.size() ? n - s.size() : 0, ' '); };
    line("numero de Rayleigh                    ", fg(P.Ra));
    line("numero de Prandtl                     ", fg(P.Pr));
    line("incremento de tiempo                  ", fg(P.dt));
    line("iteraciones maximas                   ", fi(P.itermax));
    line("paquete de iteraciones                ", fi(P.paq_itera));
    line("numero de Richardson                  ", fg(P.Ri_1));
    line("relajacion de la presion              ", fg(P.rel_pres));
    line("relajacion de la velocidad            ", fg(P.rel_vel));
    line("relajacion de la temperatura          ", fg(P.rel_ener));
    line("convergencia de la velocidad          ", fg(P.conv_u));
    line("convergencia de la temperatura        ", fg(P.conv_t));
    line("convergencia de la presion            ", fg(P.conv_p));
    line("convergencia del residuo              ", fg(P.conv_resi));
    line("convergencia del paso de tiempo       ", fg(P.conv_paso));
    line("iteraciones maximas de SIMPLE         ", fi(P.iter_simple_max));
    line("iteraciones maximas de las ecuaciones ", fi(P.iter_ecuaci_max));
    line("archivo de entrada para u             ", " " + pad(P.entrada_u, 28));
    line("archivo de entrada para v             ", " " + pad(P.entrada_v, 28));
    line("archivo de entrada para t y p         ", " " + pad(P.entrada_tp, 28));
    line("opcion de flujo inicial               ", " " + pad(P.flujo_ini, 8));
    line("opcion de temperatura inicial         ", " " + pad(P.tempe_ini, 8));
    std::fclose(f);
  }

  if (say) std::printf(" Inicia lectura de mallas\n");
  {
    const int st = ixb_read_state_files(P.entrada_u.c_str(), P.entrada_v.c_str(), P.entrada_tp.c_str(), mi, nj,
                                        xu.data(), yv.data(), xp.data(), yp.data(), u_ant.data(), v_ant.data(),
                                        T_ant.data(), p.data(), &placa_min, &placa_max, &itera_inicial, &ao);
    if (st != IXB_OK) die(2, std::string("reading the mesh files: ") + ixb_strerror(st));
  }
  if (say) std::printf(" Finaliza lectura de mallas\n --------------------------\n");
  const double tiempo_inicial = itera_inicial * P.dt;
  // condicion_inicial_flujo / condicion_inicial_tempe; other options keep the file's fields
  if (P.flujo_ini == "nulo") {
    std::fill(u_ant.begin(), u_ant.end(), 0.0);
    std::fill(v_ant.begin(), v_ant.end(), 0.0);
  }
  if (P.tempe_ini == "baja") std::fill(T_ant.begin(), T_ant.end(), 0.0);
  else if (P.tempe_ini == "alta") std::fill(T_ant.begin(), T_ant.end(), 1.0);
  u = u_ant;
  v = v_ant;
  T = T_ant;

  {
    int st = ixb_read_bc_file("cond_fronterau.dat", xu.data(), mi, yp.data(), nj + 1, bcu);
    if (st != IXB_OK) die(2, std::string("cond_fronterau.dat: ") + ixb_strerror(st));
    st = ixb_read_bc_file("cond_fronterav.dat", xp.data(), mi + 1, yv.data(), nj, bcv);
    if (st != IXB_OK) die(2, std::string("cond_fronterav.dat: ") + ixb_strerror(st));
    st = ixb_read_bc_file("cond_fronterat.dat", xp.data(), mi + 1, yp.data(), nj + 1, bct);
    if (st != IXB_OK) die(2, std::string("cond_fronterat.dat: ") + ixb_strerror(st));
  }

  // definir_cuerpo: penalty sources of the chosen body ('sincu': none)
  std::vector<double> fcu, flu, fcv, flv, fct, flt;
  if (opt.cuerpo >= 0) {
    fcu.assign(NU, 0.0); flu.assign(NU, 0.0);
    fcv.assign(NV, 0.0); flv.assign(NV, 0.0);
    fct.assign(NP, 0.0); flt.assign(NP, 0.0);
    ck(ixb_body_sources(mi, nj, xp.data(), yp.data(), opt.cuerpo, nullptr, 0, 0.0, fcu.data(), flu.data(),
                        fcv.data(), flv.data(), fct.data(), flt.data()),
       "ixb_body_sources");
  }

  ixb_params prm{};
  prm.gamma_momen = gamma_momen;
  prm.gamma_energ = gamma_energ;
  prm.Ri = Ri;
  prm.Riy = Riy;
  prm.dt = P.dt;
  prm.rel_vel = P.rel_vel;
  prm.rel_pres = P.rel_pres;
  prm.rel_ener = P.rel_ener;
  prm.conv_u = P.conv_u;
  prm.conv_p = P.conv_p;
  prm.conv_t = P.conv_t;
  prm.conv_resi = P.conv_resi;
  prm.conv_paso = P.conv_paso;
  prm.p_update = 0.6;
  prm.iter_ecuaci_max = P.iter_ecuaci_max;
  prm.iter_simple_max = P.iter_simple_max;
  prm.solver = opt.solver;

  if (opt.check) {
    std::printf("mi=%d\nnj=%d\nRec=%s\nadimen=%s\n", mi, nj, Rec.c_str(), P.adimen.c_str());
    std::printf("gamma_momen=%.17g\ngamma_energ=%.17g\nRi=%.17g\nRiy=%.17g\ndt=%.17g\n", gamma_momen, gamma_energ, Ri,
                Riy, P.dt);
    std::printf("rel_pres=%.17g\nrel_vel=%.17g\nrel_ener=%.17g\n", P.rel_pres, P.rel_vel, P.rel_ener);
    std::printf("conv_u=%.17g\nconv_t=%.17g\nconv_p=%.17g\nconv_resi=%.17g\nconv_paso=%.17g\n", P.conv_u, P.conv_t,
                P.conv_p, P.conv_resi, P.conv_paso);
    std::printf("paq_itera=%d\nitermax=%d\niter_ecuaci_max=%d\niter_simple_max=%d\npostprocesar=%d\n", P.paq_itera,
                P.itermax, P.iter_ecuaci_max, P.iter_simple_max, P.postprocesar);
    std::printf("entrada_u=%s\nentrada_v=%s\nentrada_tp=%s\nflujo_ini=%s\ntempe_ini=%s\n", P.entrada_u.c_str(),
                P.entrada_v.c_str(), P.entrada_tp.c_str(), P.flujo_ini.c_str(), P.tempe_ini.c_str());
    std::printf("placa_min=%d\nplaca_max=%d\nitera_inicial=%d\nao=%.17g\n", placa_min, placa_max, itera_inicial, ao);
    std::printf("nusselt_file=nuss_sim_%s.dat\nfolder=%s\n", tag.c_str(), folder.c_str());
    for (int s = 0; s < 4; ++s) std::printf("bc_t_side%d_ndivis=%d\n", s, bct[s].ndivis);
    return 0;
  }

  ixb_handle* h = nullptr;
  ck(ixb_create(mi, nj, opt.prec, &h), "ixb_create");
  ck(ixb_set_mesh(h, xu.data(), yv.data(), xp.data(), yp.data()), "ixb_set_mesh");
  ck(ixb_set_params(h, &prm), "ixb_set_params");
  ck(ixb_set_bc(h, IXB_VAR_U, bcu), "ixb_set_bc(u)");
  ck(ixb_set_bc(h, IXB_VAR_V, bcv), "ixb_set_bc(v)");
  ck(ixb_set_bc(h, IXB_VAR_T, bct), "ixb_set_bc(T)");
  if (opt.cuerpo >= 0) {
    ck(ixb_set_sources(h, IXB_VAR_U, fcu.data(), flu.data()), "ixb_set_sources(u)");
    ck(ixb_set_sources(h, IXB_VAR_V, fcv.data(), flv.data()), "ixb_set_sources(v)");
    ck(ixb_set_sources(h, IXB_VAR_T, fct.data(), flt.data()), "ixb_set_sources(T)");
  }
  ck(ixb_upload_state(h, u.data(), v.data(), p.data(), T.data(), u_ant.data(), v_ant.data(), T_ant.data()),
     "ixb_upload_state");
  if (opt.autotune) ck(ixb_autotune(h, 3, 0, nullptr, nullptr), "ixb_autotune");

  if (say) {
    std::printf(" IXCHEL2D: Doble : kind=  8, Precision= 15 Rango= 307\n  \n");
    std::printf(" Re=%-6s, Pr=%8.3f, Ri=%8.3f, rel_pres=%8.3f, rel_vel=%8.3f\n", Rec.c_str(), P.Pr, P.Ri_1,
                P.rel_pres, P.rel_vel);
    std::printf(" Iteracion inicial=%7d, mi=%5d, nj=%5d\n", itera_inicial, mi, nj);
    std::printf(" No. de Eckert=%13.10f, a_ent=%15.3f\n  \n", 0.0, 0.0);
    std::fflush(stdout);
  }

  // uf, vf: velocities at the p nodes for the VTK file (main.f90:1290-1312);
  // entries the reference never writes stay 0
  std::vector<double> uf(NP, 0.0), vf(NP, 0.0);
  auto Pn = [&](std::vector<double>& a, int ii, int jj) -> double& { return a[(size_t)(jj - 1) * (mi + 1) + (ii - 1)]; };

  // pinned host buffers of the package writer (u, v, p, T in the reference's shapes)
  struct Pinned {
    double* p = nullptr;
    ~Pinned() { if (p) ixb_host_free(p); }
  } U_, V_, P_, T_;
  const size_t nu_ = (size_t)mi * (nj + 1), nv_ = (size_t)(mi + 1) * nj;
  ck(ixb_host_alloc(nu_ * sizeof(double), (void**)&U_.p), "ixb_host_alloc");
  ck(ixb_host_alloc(nv_ * sizeof(double), (void**)&V_.p), "ixb_host_alloc");
  ck(ixb_host_alloc(NP * sizeof(double), (void**)&P_.p), "ixb_host_alloc");
  ck(ixb_host_alloc(NP * sizeof(double), (void**)&T_.p), "ixb_host_alloc");
  auto WU = [&](int ii, int jj) -> double { return U_.p[(size_t)(jj - 1) * mi + (ii - 1)]; };
  auto WV = [&](int ii, int jj) -> double { return V_.p[(size_t)(jj - 1) * (mi + 1) + (ii - 1)]; };
  auto WP = [&](int ii, int jj) -> double { return P_.p[(size_t)(jj - 1) * (mi + 1) + (ii - 1)]; };
  auto WT = [&](int ii, int jj) -> double { return T_.p[(size_t)(jj - 1) * (mi + 1) + (ii - 1)]; };
  std::thread writer;
  std::string writer_error;
  auto join_writer = [&]() {
    if (writer.joinable()) writer.join();
    if (!writer_error.empty()) die(3, writer_error);
  };

  int itera = 0;
  double nusselt0 = 0.0, nusselt1 = 0.0, maxbo = 0.0, residuo = 0.0;
  int64_t simple_total = 0, limit_hits = 0, momen_total = 0, pres_total = 0, ener_total = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int ll = 1; ll <= P.itermax / P.paq_itera; ++ll) {
    for (int kk = 1; kk <= P.paq_itera; ++kk) {
      ixb_report rep{};
      const int st = ixb_step(h, &rep);
      if (st != IXB_OK)
        die(3, "ixb_step at time step " + std::to_string(itera_inicial + itera + 1) + ": " + ixb_strerror(st));
      maxbo = rep.maxbo;
      residuo = rep.residuo;
      simple_total += rep.n_simple;
      momen_total += rep.n_momen;
      pres_total += rep.n_pres;
      ener_total += rep.n_ener;
      if (rep.exit_code == 2) ++limit_hits;
      ++itera;
      if (say && itera % 500 == 0)
        std::printf(" ITERACION: %s%s%s\n", fi(itera).c_str(), fg(residuo).c_str(), fg(maxbo).c_str());
      if (itera % 1000 == 0) {
        ck(ixb_nusselt_y(h, placa_min, placa_max, &nusselt0, &nusselt1), "ixb_nusselt_y");
        ck(ixb_download_state(h, nullptr, nullptr, nullptr, T.data(), nullptr, nullptr, nullptr),
           "ixb_download_state");
        const int ic = (placa_min + placa_max) / 2, jc = nj / 2 + 1;
        const double temp_med = (Pn(T, ic, jc) + Pn(T, ic + 1, jc)) / 2.0;
        const std::string name = "nuss_sim_" + tag + ".dat";
        FILE* f = std::fopen(name.c_str(), "a");
        if (!f) die(3, "cannot open " + name);
        std::fprintf(f, "%s%s%s%s%s%s\n", fmt_d23_15(tiempo_inicial + itera * P.dt).c_str(),
                     fmt_d23_15(nusselt0).c_str(), fmt_d23_15(-nusselt1).c_str(), fmt_d23_15(temp_med).c_str(),
                     fmt_d23_15(0.0).c_str(), fmt_d23_15(0.0).c_str());
        std::fclose(f);
      }
    }
    const int itera_total = itera_inicial + itera;
    const int q = P.paq_itera;
    const int millar = itera_total / (1000 * q);
    const int centena = (itera_total - millar * 1000 * q) / (100 * q);
    const int decena = (itera_total - millar * 1000 * q - centena * 100 * q) / (10 * q);
    const int unidad = (itera_total - millar * 1000 * q - centena * 100 * q - decena * 10 * q) / q;
    const int decima =
        q / 10 > 0 ? (itera_total - millar * 1000 * q - centena * 100 * q - decena * 10 * q - unidad * q) / (q / 10)
                   : 0;
    // the package's state goes to the writer: a snapshot on the device, copied
    // to pinned host buffers on the library's download stream while the next
    // package runs; the writer thread formats and writes the files once the
    // copies have landed.  The previous writer is joined first: it reads the
    // same host buffers.
    join_writer();
    ck(ixb_download_state_async(h, U_.p, V_.p, P_.p, T_.p, nullptr, nullptr, nullptr), "ixb_download_state_async");
    if (say) {
      std::printf(" itera_total=%s\n", fi(itera_total).c_str());
      std::printf(" N_Izq=%s, N_Der=%s\n", fmt_d23_15(nusselt0).c_str(), fmt_d23_15(nusselt1).c_str());
      std::printf(" b_o  =%s, Res_u=%s\n", fmt_d23_15(maxbo).c_str(), fmt_d23_15(residuo).c_str());
      std::printf(" Res_T=%s, Res_v=%s\n  \n", fmt_d23_15(0.0).c_str(), fmt_d23_15(0.0).c_str());
      std::fflush(stdout);
    }
    writer = std::thread([&, itera_total, millar, centena, decena, unidad, decima]() {
      if (ixb_download_wait(h) != IXB_OK) {
        writer_error = "ixb_download_wait failed";
        return;
      }
      for (int jj = 2; jj <= nj; ++jj) {
        for (int ii = 2; ii <= mi; ++ii) Pn(uf, ii, jj) = (WU(ii, jj) + WU(ii - 1, jj)) / 2.0;
        Pn(vf, 1, jj) = WV(1, jj);
        Pn(vf, mi + 1, jj) = WV(mi + 1, jj);
      }
      for (int ii = 2; ii <= mi; ++ii)
        for (int jj = 2; jj <= nj; ++jj) Pn(vf, ii, jj) = (WV(ii, jj) + WV(ii, jj - 1)) / 2.0;
      for (int jj = 1; jj <= nj + 1; ++jj) {
        Pn(uf, 1, jj) = WU(1, jj);
        Pn(uf, mi + 1, jj) = WU(mi, jj);
      }
      for (int ii = 1; ii <= mi + 1; ++ii) {
        Pn(vf, ii, 1) = WV(ii, 1);
        Pn(vf, ii, nj + 1) = WV(ii, nj);
      }
      if (!P.postprocesar) return;
      const std::string fu = "out_" + tag + "u.dat", fv = "out_" + tag + "v.dat", fp = "out_" + tag + "p.dat";
      const int st = ixb_write_state_files(fu.c_str(), fv.c_str(), fp.c_str(), mi, nj, xu.data(), yv.data(),
                                           xp.data(), yp.data(), U_.p, V_.p, T_.p, P_.p, placa_min, placa_max,
                                           itera_total, ao);
      if (st != IXB_OK) {
        writer_error = std::string("writing out_*.dat: ") + ixb_strerror(st);
        return;
      }
      // postproceso_bin: unformatted stream records, native byte order
      std::string bu, bv, bp;
      for (int jj = 1; jj <= nj + 1; ++jj)
        for (int ii = 1; ii <= mi; ++ii) put_doubles(&bu, xu[ii - 1], yp[jj - 1], WU(ii, jj));
      for (int jj = 1; jj <= nj; ++jj)
        for (int ii = 1; ii <= mi + 1; ++ii) put_doubles(&bv, xp[ii - 1], yv[jj - 1], WV(ii, jj));
      for (int jj = 1; jj <= nj + 1; ++jj)
        for (int ii = 1; ii <= mi + 1; ++ii) put_doubles(&bp, WT(ii, jj), WP(ii, jj));
      if (!write_file("out_" + tag + "u.bin", bu) || !write_file("out_" + tag + "v.bin", bv) ||
          !write_file("out_" + tag + "p.bin", bp)) {
        writer_error = "cannot write out_*.bin";
        return;
      }
      // postproceso_vtk: legacy VTK structured grid, big-endian binary
      const std::string npts = fi((int64_t)(mi + 1) * (nj + 1));
      std::string vtk;
      vtk += "# vtk DataFile Version 2.3\n3D Mesh\nBINARY\nDATASET STRUCTURED_GRID\n";
      vtk += "DIMENSIONS " + fi(mi + 1) + fi(nj + 1) + fi(1) + "\n";
      vtk += "POINTS " + npts + " float\n";
      for (int jj = 1; jj <= nj + 1; ++jj)
        for (int ii = 1; ii <= mi + 1; ++ii) {
          put_be_float(&vtk, xp[ii - 1]);
          put_be_float(&vtk, yp[jj - 1]);
          put_be_float(&vtk, 0.0);
        }
      vtk += "\nPOINT_DATA " + npts;
      vtk += "SCALARS PRESS float\nLOOKUP_TABLE default\n";
      for (size_t k = 0; k < NP; ++k) put_be_float(&vtk, P_.p[k]);
      vtk += "\nSCALARS TEMPER float\nLOOKUP_TABLE default\n";
      for (size_t k = 0; k < NP; ++k) put_be_float(&vtk, T_.p[k]);
      vtk += "\nVECTORS VELOCITY float\n";
      for (size_t k = 0; k < NP; ++k) {
        put_be_float(&vtk, uf[k]);
        put_be_float(&vtk, vf[k]);
        put_be_float(&vtk, 0.0);
      }
      const std::string vname = folder + "/t_" + std::string{digit(millar), digit(centena), digit(decena),
                                                             digit(unidad), digit(decima)} + ".vtk";
      if (!write_file(vname, vtk)) writer_error = "cannot write " + vname;
    });
  }
  join_writer();
  if (!writer_error.empty()) die(3, writer_error);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ck(ixb_destroy(h), "ixb_destroy");
  // run summary (also under --quiet): time steps, SIMPLE iterations, the
  // inner passes of the momentum / pressure-correction / energy loops, seconds
  std::printf(" pasos de tiempo=%d, iteraciones SIMPLE=%lld (limite alcanzado en %lld pasos), "
              "pases internos momento/presion/energia=%lld/%lld/%lld, %.3f s\n",
              itera, (long long)simple_total, (long long)limit_hits, (long long)momen_total, (long long)pres_total,
              (long long)ener_total, secs);
  return 0;
}
