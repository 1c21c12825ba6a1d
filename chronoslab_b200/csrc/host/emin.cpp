// Host rows of the EMIN prolongation pattern (restating the row loop of
// MEX_EMIN/MEX_cptProlPatt.cpp:356-443); the GPU kernel (emin_gpu.cu)
// computes every other row the same way.
#include <algorithm>
#include <cmath>
#include <unordered_map>

#include "host.h"

namespace chronos {

void emin_pattern_row(int i, const CsrRef &S, const CsrRef &Pc, const CsrRef &P0, int nnzr,
                      std::vector<int> &cols, std::vector<double> &vals) {
  const int64_t s0 = P0.rp[i], e0 = P0.rp[i + 1];
  const int n0 = (int)(e0 - s0);
  const int budget = std::max(0, nnzr - n0);
  cols.clear();
  vals.clear();
  auto own = [&](int c) { return std::binary_search(P0.ci + s0, P0.ci + e0, c); };
  std::vector<std::pair<int, double>> cand;       // first-seen order
  if (budget > 0) {
    std::unordered_map<int, size_t> at;
    for (int64_t ks = S.rp[i]; ks < S.rp[i + 1]; ++ks) {
      const int j = S.ci[ks];
      const double sij = S.v[ks];
      for (int64_t kp = Pc.rp[j]; kp < Pc.rp[j + 1]; ++kp) {
        const int c = Pc.ci[kp];
        if (own(c)) continue;
        auto it = at.find(c);
        if (it == at.end()) {
          at.emplace(c, cand.size());
          cand.emplace_back(c, sij * Pc.v[kp]);
        } else {
          cand[it->second].second += sij * Pc.v[kp];
        }
      }
    }
    cand.erase(std::remove_if(cand.begin(), cand.end(),
                              [](const std::pair<int, double> &cv) { return cv.second == 0.0; }),
               cand.end());
    if ((int)cand.size() > budget) {
      std::nth_element(cand.begin(), cand.begin() + budget, cand.end(),
                       [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                         const double aa = std::fabs(a.second), bb = std::fabs(b.second);
                         return aa != bb ? aa > bb : a.first < b.first;
                       });
      cand.resize(budget);
    }
  }
  for (int64_t k = s0; k < e0; ++k) cand.emplace_back(P0.ci[k], 1.0);
  std::sort(cand.begin(), cand.end(),
            [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
              return a.first < b.first;
            });
  for (const auto &cv : cand) {
    cols.push_back(cv.first);
    vals.push_back(cv.second);
  }
}

}  // namespace chronos
