// Matrix Market coordinate files -> CSR in full storage (trl_csr_read_mtx, trl_solver.h).
//
// Semantics of the reference's loader (examples/sycl/csrevp.hh:26-124): the header line
// "%%MatrixMarket ..." is matched case-insensitively and "symmetric" in it mirrors every
// off-diagonal entry (i, j) as (j, i), placed right after it; indices are 1-based; the CSR
// is built by a counting sort on the row that keeps, within a row, the order in which the
// entries (mirrors included) were read; duplicates are kept. Beyond it: "pattern" files
// (no value column) get 1.0, "integer" values are read as doubles, and malformed input is
// reported instead of read as garbage.
//
// The data lines are parsed by several host threads, each on a byte range that starts at
// a line boundary; their entries are concatenated in file order before the row sort.
#include "trl_solver.h"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace trl_solver_detail {
int set_error(int status, const char* msg); // records trl_solver_last_error (solver_capi.cc)
}

namespace {

using trl_solver_detail::set_error;

struct Entries {
  std::vector<int64_t> row, col; // 0-based
  std::vector<double> val;
  std::string error;
};

const char* skip_space(const char* p, const char* end)
{
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  return p;
}

// Parses the entry lines in [p, end); `pattern`: no value column.
void parse_range(const char* p, const char* end, bool pattern, bool symmetric, int64_t n_rows, int64_t n_cols, Entries& out)
{
  while (p < end) {
    p = skip_space(p, end);
    if (p == end) break;
    if (*p == '\n') {
      ++p;
      continue;
    }
    if (*p == '%') { // comment line
      while (p < end && *p != '\n') ++p;
      continue;
    }
    int64_t r = 0, c = 0;
    double v = 1.0;
    auto res = std::from_chars(p, end, r);
    if (res.ec != std::errc()) {
      out.error = "bad row index";
      return;
    }
    p = skip_space(res.ptr, end);
    res = std::from_chars(p, end, c);
    if (res.ec != std::errc()) {
      out.error = "bad column index";
      return;
    }
    p = res.ptr;
    if (!pattern) {
      p = skip_space(p, end);
      if (p < end && *p == '+') ++p; // from_chars takes no leading '+'; stream extraction does
      auto rv = std::from_chars(p, end, v);
      if (rv.ec != std::errc()) {
        out.error = "bad value";
        return;
      }
      p = rv.ptr;
    }
    while (p < end && *p != '\n') ++p; // ignore the rest of the line
    if (r < 1 || r > n_rows || c < 1 || c > n_cols) {
      out.error = "index out of range";
      return;
    }
    out.row.push_back(r - 1);
    out.col.push_back(c - 1);
    out.val.push_back(v);
    if (symmetric && r != c) {
      out.row.push_back(c - 1);
      out.col.push_back(r - 1);
      out.val.push_back(v);
    }
  }
}

std::string lower(std::string s)
{
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char ch) { return static_cast<char>(std::tolower(ch)); });
  return s;
}

} // namespace

extern "C" int trl_csr_read_mtx(const char* path, int threads, int64_t* n_rows, int64_t* n_cols, int64_t* nnz, int32_t** rowptr, int32_t** colind, double** values)
{
  if (!path || !n_rows || !n_cols || !nnz || !rowptr || !colind || !values) return set_error(TRL_EINVAL, "null argument");
  *rowptr = nullptr;
  *colind = nullptr;
  *values = nullptr;
  std::FILE* f = std::fopen(path, "rb");
  if (!f) return set_error(TRL_EINVAL, (std::string("cannot open ") + path).c_str());
  std::string buf;
  {
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.append(chunk, got);
    std::fclose(f);
  }
  const char* p = buf.data();
  const char* end = p + buf.size();
  // header and comments up to the size line
  bool symmetric = false, pattern = false;
  const char* line = p;
  while (line < end) {
    const char* eol = static_cast<const char*>(std::memchr(line, '\n', static_cast<size_t>(end - line)));
    if (!eol) eol = end;
    const char* q = skip_space(line, eol);
    if (q == eol) { // blank line
      line = eol + (eol < end);
      continue;
    }
    if (*q == '%') {
      const std::string h = lower(std::string(q, eol));
      if (h.rfind("%%matrixmarket", 0) == 0) {
        if (h.find("coordinate") == std::string::npos) return set_error(TRL_EINVAL, "only coordinate Matrix Market files are supported");
        if (h.find("complex") != std::string::npos || h.find("hermitian") != std::string::npos || h.find("skew") != std::string::npos)
          return set_error(TRL_EINVAL, "complex, hermitian and skew-symmetric files are not supported");
        symmetric = h.find("symmetric") != std::string::npos;
        pattern = h.find("pattern") != std::string::npos;
      }
      line = eol + (eol < end);
      continue;
    }
    break;
  }
  if (line >= end) return set_error(TRL_EINVAL, "no size line");
  int64_t rows = 0, cols = 0, entries = 0;
  {
    const char* eol = static_cast<const char*>(std::memchr(line, '\n', static_cast<size_t>(end - line)));
    if (!eol) eol = end;
    const char* q = skip_space(line, eol);
    auto a = std::from_chars(q, eol, rows);
    auto b = a.ec == std::errc() ? std::from_chars(skip_space(a.ptr, eol), eol, cols) : a;
    auto c = b.ec == std::errc() ? std::from_chars(skip_space(b.ptr, eol), eol, entries) : b;
    if (a.ec != std::errc() || b.ec != std::errc() || c.ec != std::errc() || rows < 0 || cols < 0 || entries < 0)
      return set_error(TRL_EINVAL, "bad size line");
    line = eol + (eol < end);
  }
  // split the data region at line boundaries
  const int64_t bytes = end - line;
  int T = threads > 0 ? threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  T = static_cast<int>(std::min<int64_t>(T, std::max<int64_t>(1, bytes / (1 << 20)))); // at least 1 MiB per thread
  std::vector<const char*> cut(T + 1);
  cut[0] = line;
  cut[T] = end;
  for (int t = 1; t < T; ++t) {
    const char* q = line + bytes * t / T;
    if (q < cut[t - 1]) q = cut[t - 1];
    const char* nl = static_cast<const char*>(std::memchr(q, '\n', static_cast<size_t>(end - q)));
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<Entries> parts(T);
  {
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(parse_range, cut[t], cut[t + 1], pattern, symmetric, rows, cols, std::ref(parts[t]));
    parse_range(cut[0], cut[1], pattern, symmetric, rows, cols, parts[0]);
    for (auto& th : pool) th.join();
  }
  int64_t total = 0;
  for (const auto& e : parts) {
    if (!e.error.empty()) return set_error(TRL_EINVAL, e.error.c_str());
    total += static_cast<int64_t>(e.row.size());
  }
  // entries in the file: count without the mirrors
  int64_t in_file = 0;
  for (const auto& e : parts) {
    size_t i = 0;
    while (i < e.row.size()) {
      const bool mirrored = symmetric && e.row[i] != e.col[i];
      i += mirrored ? 2 : 1;
      ++in_file;
    }
  }
  if (in_file != entries) return set_error(TRL_EINVAL, "number of entries differs from the size line");
  if (total >= (int64_t(1) << 31) || rows >= (int64_t(1) << 31)) return set_error(TRL_EINVAL, "matrix too large for int32 CSR indices");
  // counting sort on the row, stable
  int32_t* rp = static_cast<int32_t*>(std::calloc(static_cast<size_t>(rows) + 1, sizeof(int32_t)));
  int32_t* ci = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * static_cast<size_t>(std::max<int64_t>(total, 1))));
  double* va = static_cast<double*>(std::malloc(sizeof(double) * static_cast<size_t>(std::max<int64_t>(total, 1))));
  if (!rp || !ci || !va) {
    std::free(rp);
    std::free(ci);
    std::free(va);
    return set_error(TRL_ENOMEM, "host allocation failed");
  }
  for (const auto& e : parts)
    for (int64_t r : e.row) ++rp[r + 1];
  for (int64_t i = 0; i < rows; ++i) rp[i + 1] += rp[i];
  std::vector<int32_t> pos(rp, rp + rows);
  for (const auto& e : parts)
    for (size_t i = 0; i < e.row.size(); ++i) {
      const int32_t at = pos[e.row[i]]++;
      ci[at] = static_cast<int32_t>(e.col[i]);
      va[at] = e.val[i];
    }
  *n_rows = rows;
  *n_cols = cols;
  *nnz = total;
  *rowptr = rp;
  *colind = ci;
  *values = va;
  return TRL_OK;
}

extern "C" void trl_csr_free_host(int32_t* rowptr, int32_t* colind, double* values)
{
  std::free(rowptr);
  std::free(colind);
  std::free(values);
}
