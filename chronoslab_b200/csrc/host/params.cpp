// Parameter files of the reference: aspAMG.fnames names seven positional
// files, one value per line (first token; the rest is a '%' comment).
// Restates readDefaultParams.m:1-31, aspAMG_main.m:17-59 and read_amg.m,
// read_smoother.m:73-79, read_tspace.m, read_coarsen.m:177-179,
// read_prolong.m:3-26, read_filter.m:3-14, read_general.m:4-11.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "host.h"
#include "../errors.h"

namespace chronos {
namespace {

std::vector<std::string> first_tokens(const std::string &path, size_t n) {
  std::ifstream f(path);
  if (!f) throw Error(CHRONOS_EIO, "cannot open parameter file " + path);
  std::vector<std::string> out;
  std::string line;
  while (out.size() < n && std::getline(f, line)) {
    std::istringstream ss(line);
    std::string tok;
    ss >> tok;
    out.push_back(tok);
  }
  if (out.size() < n)
    throw Error(CHRONOS_EIO, path + ": expected " + std::to_string(n) + " lines");
  return out;
}

double num(const std::string &t, const std::string &file) {
  char *end = nullptr;
  double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) throw Error(CHRONOS_EIO, file + ": bad number '" + t + "'");
  return v;
}

void copy_str(char *dst, size_t cap, const std::string &s) {
  std::snprintf(dst, cap, "%s", s.c_str());
}

bool truthy(std::string s) {
  for (auto &c : s) c = (char)tolower(c);
  return s == "true" || s == "1";
}

}  // namespace

void params_default(chronos_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->nLevMax = 10;
  p->maxCoarseSZ = 1000;
  p->nthread = 0;                    // 0: all host threads
  p->nupre = 1;
  p->nupost = 1;
  p->nstep = 15;
  p->step_size = 1;
  p->epsilon = 1e-3;
  copy_str(p->smoother_method, sizeof p->smoother_method, "AFSAI_SYM");
  p->ntv = 6;
  p->tspace_itmax = 40;
  p->tspace_tol = 1e-4;
  copy_str(p->tspace_method, sizeof p->tspace_method, "NONE");
  p->init_approx = 5;
  copy_str(p->SoC_type, sizeof p->SoC_type, "DOM");
  p->soc_tau = 0.01;
  p->nl_agg = 0;
  copy_str(p->proltype, sizeof p->proltype, "BAMG");
  copy_str(p->prol_emin, sizeof p->prol_emin, "NONE");
  p->prol_np = 0;
  p->itmax_vol = 100;
  p->tol_vol = 0.01;
  p->dist_min = 1;
  p->dist_max = 10;
  p->maxcond = 1e13;
  p->maxrownrm = 5.0;
  p->eps_prol = 1e-10;
  p->updateCF = 0;
  p->patt_pow = 2;
  p->patt_tau = 0.01;
  p->nnzr_max = 30;
  p->itmax_emin = 10;
  p->energ_tol = 1e-3;
  p->condmax_emin = 1e10;
  p->prec_emin = 1;
  p->solv_emin = 4;
  p->filt_np = 0;
  p->filt_wgt = 170.0;
  p->filt_tol = 0.1;
  p->filt_tau = 0.0;
  p->min_patt = 0;
  p->ascii_input = 0;
  copy_str(p->rhs_build, sizeof p->rhs_build, "unit_rhs");
  p->symmetric = 1;
  copy_str(p->solv_method, sizeof p->solv_method, "PCG");
  p->itmax = 15000;
  p->tol = 1e-8;
  p->restart = 100;
  p->precision = CHRONOS_FP32;
  p->use_graph = 1;
  p->seed = 5489;
  p->fsai_fabs = 0;
  p->use_bsr = 1;
  p->exact_outer = 0;
  p->replace_ratio = 0.01;
  p->spmv_format = 0;
  p->batch_grouped = 1;
}

void params_read(const char *fnames_path, chronos_params *p) {
  std::string fp(fnames_path);
  std::string dir = ".";
  auto slash = fp.find_last_of('/');
  if (slash != std::string::npos) dir = fp.substr(0, slash);
  auto names = first_tokens(fp, 7);
  auto path = [&](int k) { return names[k][0] == '/' ? names[k] : dir + "/" + names[k]; };
  auto amg = first_tokens(path(0), 2);
  p->nLevMax = (int)num(amg[0], path(0));
  p->maxCoarseSZ = (int)num(amg[1], path(0));
  auto smo = first_tokens(path(1), 7);
  p->nthread = (int)num(smo[0], path(1));
  p->nupre = (int)num(smo[1], path(1));
  p->nupost = (int)num(smo[2], path(1));
  p->nstep = (int)num(smo[3], path(1));
  p->step_size = (int)num(smo[4], path(1));
  p->epsilon = num(smo[5], path(1));
  copy_str(p->smoother_method, sizeof p->smoother_method, smo[6]);
  auto tsp = first_tokens(path(2), 5);
  p->ntv = (int)num(tsp[0], path(2));
  p->tspace_itmax = (int)num(tsp[1], path(2));
  p->tspace_tol = num(tsp[2], path(2));
  copy_str(p->tspace_method, sizeof p->tspace_method, tsp[3]);
  p->init_approx = (int)num(tsp[4], path(2));
  auto coa = first_tokens(path(3), 3);
  copy_str(p->SoC_type, sizeof p->SoC_type, coa[0]);
  p->soc_tau = num(coa[1], path(3));
  p->nl_agg = (int)num(coa[2], path(3));
  auto pro = first_tokens(path(4), 22);
  copy_str(p->proltype, sizeof p->proltype, pro[0]);
  copy_str(p->prol_emin, sizeof p->prol_emin, pro[1]);
  p->prol_np = (int)num(pro[2], path(4));
  p->itmax_vol = (int)num(pro[3], path(4));
  p->tol_vol = num(pro[4], path(4));
  p->dist_min = (int)num(pro[5], path(4));
  p->dist_max = (int)num(pro[6], path(4));
  p->maxcond = num(pro[7], path(4));
  p->maxrownrm = num(pro[8], path(4));
  p->eps_prol = num(pro[9], path(4));
  p->updateCF = (int)num(pro[10], path(4));
  p->patt_pow = (int)num(pro[11], path(4));
  p->patt_tau = num(pro[12], path(4));
  p->nnzr_max = (int)num(pro[13], path(4));
  p->itmax_emin = (int)num(pro[14], path(4));
  p->energ_tol = num(pro[15], path(4));
  p->condmax_emin = num(pro[16], path(4));
  p->prec_emin = (int)num(pro[17], path(4));
  p->solv_emin = (int)num(pro[18], path(4));
  auto fil = first_tokens(path(5), 5);
  p->filt_np = (int)num(fil[0], path(5));
  p->filt_wgt = num(fil[1], path(5));
  p->filt_tol = num(fil[2], path(5));
  p->filt_tau = num(fil[3], path(5));
  p->min_patt = (int)num(fil[4], path(5));
  auto gen = first_tokens(path(6), 7);
  p->ascii_input = truthy(gen[0]) ? 1 : 0;
  copy_str(p->rhs_build, sizeof p->rhs_build, gen[1]);
  p->symmetric = truthy(gen[2]) ? 1 : 0;
  copy_str(p->solv_method, sizeof p->solv_method, gen[3]);
  p->itmax = (int)num(gen[4], path(6));
  p->tol = num(gen[5], path(6));
  p->restart = (int)num(gen[6], path(6));
}

}  // namespace chronos
