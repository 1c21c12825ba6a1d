// On-disk matrix formats of the reference, read and written on the host.
//
//  * example_cpp binary CSR (Cpp_EMIN/readMat.cpp:4-80): a header of two
//    int32 (rows, entries), then one 16-byte record per entry {int32 row,
//    int32 column, float64 value}, 1-based, entries grouped by ascending row;
//    square matrices.
//  * Chronos .Ext_bin (debug_stuff/dump_chronos/DumpChronos.cpp:27-45): the
//    matrix file holds int64 rows, int64 entries, then one 24-byte record per
//    entry {int64 row, int64 column, float64 value} (1-based, as MATLAB's
//    find writes them); the test-space file holds int64 rows, int64 columns,
//    then the values row by row.  (The reference's dumper writes the values
//    of the test space into the matrix file it has just closed, so its test
//    space files end after the header; the reader accepts that and returns
//    zero columns of values.)
// Entries are returned as a 0-based CSR with each row's columns ascending
// (duplicates summed in file order).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>

#include "../errors.h"
#include "host.h"

namespace chronos {

namespace {

struct File {
  FILE *f = nullptr;
  File(const std::string &path, const char *mode) : f(std::fopen(path.c_str(), mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// Bytes left from the current position to the end of the file.
int64_t bytes_left(FILE *f) {
  const long here = std::ftell(f);
  if (here < 0 || std::fseek(f, 0, SEEK_END) != 0) return -1;
  const long end = std::ftell(f);
  std::fseek(f, here, SEEK_SET);
  return end < here ? -1 : (int64_t)(end - here);
}

template <typename T>
bool read_one(FILE *f, T &v) {
  return std::fread(&v, sizeof(T), 1, f) == 1;
}

// COO (0-based) to CSR with sorted rows, duplicates summed in input order.
HostCSR coo_to_csr(int nrows, int ncols, const std::vector<int> &ri, const std::vector<int> &cj,
                   const std::vector<double> &v) {
  const size_t nt = ri.size();
  std::vector<size_t> order(nt);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    return ri[a] != ri[b] ? ri[a] < ri[b] : cj[a] < cj[b];
  });
  HostCSR h;
  h.nrows = nrows;
  h.ncols = ncols;
  h.rp.assign((size_t)nrows + 1, 0);
  for (size_t q = 0; q < nt;) {
    const size_t k = order[q];
    double s = v[k];
    size_t r = q + 1;
    while (r < nt && ri[order[r]] == ri[k] && cj[order[r]] == cj[k]) s += v[order[r++]];
    h.ci.push_back(cj[k]);
    h.v.push_back(s);
    h.rp[(size_t)ri[k] + 1] += 1;
    q = r;
  }
  for (int i = 0; i < nrows; ++i) h.rp[(size_t)i + 1] += h.rp[i];
  return h;
}

}  // namespace

HostCSR read_matrix_bin(const std::string &path) {
  File fl(path, "rb");
  CHRONOS_REQUIRE(fl.f, CHRONOS_EIO, "cannot open " + path);
  int32_t nr = 0, nt = 0;
  CHRONOS_REQUIRE(read_one(fl.f, nr) && read_one(fl.f, nt) && nr >= 0 && nt >= 0, CHRONOS_EIO,
                  path + ": bad header");
  CHRONOS_REQUIRE(bytes_left(fl.f) >= (int64_t)nt * 16, CHRONOS_EIO,
                  path + ": shorter than its " + std::to_string(nt) + " entries");
  std::vector<int> ri(nt), cj(nt);
  std::vector<double> v(nt);
  for (int32_t k = 0; k < nt; ++k) {
    struct {
      int32_t ii, jj;
      double aa;
    } rec;
    static_assert(sizeof(rec) == 16, "16-byte records");
    CHRONOS_REQUIRE(std::fread(&rec, sizeof(rec), 1, fl.f) == 1, CHRONOS_EIO,
                    path + ": truncated at entry " + std::to_string(k + 1));
    CHRONOS_REQUIRE(rec.ii >= 1 && rec.ii <= nr && rec.jj >= 1 && rec.jj <= nr, CHRONOS_EIO,
                    path + ": index out of range at entry " + std::to_string(k + 1));
    ri[k] = rec.ii - 1;
    cj[k] = rec.jj - 1;
    v[k] = rec.aa;
  }
  return coo_to_csr(nr, nr, ri, cj, v);
}

HostCSR read_ext_bin(const std::string &path) {
  File fl(path, "rb");
  CHRONOS_REQUIRE(fl.f, CHRONOS_EIO, "cannot open " + path);
  int64_t nr = 0, nt = 0;
  CHRONOS_REQUIRE(read_one(fl.f, nr) && read_one(fl.f, nt) && nr >= 0 && nt >= 0 &&
                      nr < INT32_MAX && nt < INT32_MAX,
                  CHRONOS_EIO, path + ": bad header");
  CHRONOS_REQUIRE(bytes_left(fl.f) >= nt * 24, CHRONOS_EIO,
                  path + ": shorter than its " + std::to_string(nt) + " entries");
  std::vector<int> ri(nt), cj(nt);
  std::vector<double> v(nt);
  int64_t maxc = 0;
  for (int64_t k = 0; k < nt; ++k) {
    int64_t i = 0, j = 0;
    double a = 0.0;
    CHRONOS_REQUIRE(read_one(fl.f, i) && read_one(fl.f, j) && read_one(fl.f, a), CHRONOS_EIO,
                    path + ": truncated at entry " + std::to_string(k + 1));
    CHRONOS_REQUIRE(i >= 1 && i <= nr && j >= 1 && j < INT32_MAX, CHRONOS_EIO,
                    path + ": index out of range at entry " + std::to_string(k + 1));
    ri[k] = (int)(i - 1);
    cj[k] = (int)(j - 1);
    v[k] = a;
    maxc = std::max(maxc, j);
  }
  return coo_to_csr((int)nr, (int)std::max<int64_t>(nr, maxc), ri, cj, v);
}

void write_ext_bin(const std::string &path, const HostCSR &A) {
  File fl(path, "wb");
  CHRONOS_REQUIRE(fl.f, CHRONOS_EIO, "cannot open " + path + " for writing");
  const int64_t nr = A.nrows, nt = A.nnz();
  bool ok = std::fwrite(&nr, sizeof nr, 1, fl.f) == 1 && std::fwrite(&nt, sizeof nt, 1, fl.f) == 1;
  for (int i = 0; i < A.nrows && ok; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1] && ok; ++k) {
      const int64_t ii = i + 1, jj = (int64_t)A.ci[k] + 1;
      ok = std::fwrite(&ii, sizeof ii, 1, fl.f) == 1 && std::fwrite(&jj, sizeof jj, 1, fl.f) == 1 &&
           std::fwrite(&A.v[k], sizeof(double), 1, fl.f) == 1;
    }
  CHRONOS_REQUIRE(ok, CHRONOS_EIO, path + ": write failed");
}

void read_tv_ext_bin(const std::string &path, int *nrows, int *ntv, std::vector<double> &tv) {
  File fl(path, "rb");
  CHRONOS_REQUIRE(fl.f, CHRONOS_EIO, "cannot open " + path);
  int64_t nr = 0, nc = 0;
  CHRONOS_REQUIRE(read_one(fl.f, nr) && read_one(fl.f, nc) && nr >= 0 && nc >= 0 &&
                      nr < INT32_MAX && nc < 1024,
                  CHRONOS_EIO, path + ": bad header");
  *nrows = (int)nr;
  const int64_t left = bytes_left(fl.f);
  CHRONOS_REQUIRE(left == 0 || left >= nr * nc * 8, CHRONOS_EIO, path + ": truncated test space");
  std::vector<double> rowmajor(left == 0 ? 0 : (size_t)nr * nc);
  const size_t got =
      rowmajor.empty() ? 0 : std::fread(rowmajor.data(), sizeof(double), rowmajor.size(), fl.f);
  if (got == 0) {                  // header only (the reference dumper's files)
    *ntv = 0;
    tv.clear();
    return;
  }
  CHRONOS_REQUIRE(got == rowmajor.size(), CHRONOS_EIO, path + ": truncated test space");
  *ntv = (int)nc;
  tv.assign(rowmajor.size(), 0.0);      // column-major n x ntv
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t j = 0; j < nc; ++j) tv[(size_t)j * nr + i] = rowmajor[(size_t)i * nc + j];
}

void write_tv_ext_bin(const std::string &path, int nrows, int ntv, const double *tv_colmajor) {
  File fl(path, "wb");
  CHRONOS_REQUIRE(fl.f, CHRONOS_EIO, "cannot open " + path + " for writing");
  const int64_t nr = nrows, nc = ntv;
  bool ok = std::fwrite(&nr, sizeof nr, 1, fl.f) == 1 && std::fwrite(&nc, sizeof nc, 1, fl.f) == 1;
  for (int64_t i = 0; i < nr && ok; ++i)
    for (int64_t j = 0; j < nc && ok; ++j)
      ok = std::fwrite(tv_colmajor + j * nr + i, sizeof(double), 1, fl.f) == 1;
  CHRONOS_REQUIRE(ok, CHRONOS_EIO, path + ": write failed");
}

}  // namespace chronos
