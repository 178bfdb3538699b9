// Matrix loaders behind the C ABI: Matrix Market coordinate files and the
// reference's IJA triplet files, parsed on the host into CSR (duplicates
// summed, columns sorted within each row), then handed to krans_csr_create.
//
// Reference: src/IO/MatrixLoader.cpp:12-56 (load_matrix_market through
// Eigen::loadMarket; load_ija_triplet_matrix: header "rows cols nnz", then
// 0-based "i j v" triplets up to the end of the file, a warning on a count
// mismatch, duplicates summed by setFromTriplets).
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "kr_internal.h"

namespace {

using kr::set_error;

struct Triplets {
  int64_t m = 0, n = 0;
  std::vector<int64_t> i, j;
  std::vector<double> v;
};

bool read_file(const char *path, std::string &buf) {
  FILE *f = fopen(path, "rb");
  if (!f)
    return false;
  char tmp[1 << 16];
  size_t got;
  while ((got = fread(tmp, 1, sizeof tmp, f)) > 0)
    buf.append(tmp, got);
  fclose(f);
  return true;
}

// cursor over a text buffer: integers and reals separated by white space
struct Scan {
  const char *p, *end;
  void skip_ws() {
    while (p < end && isspace((unsigned char)*p))
      p++;
  }
  bool at_end() {
    skip_ws();
    return p >= end;
  }
  bool int64(int64_t &x) {
    skip_ws();
    if (p >= end)
      return false;
    char *e = nullptr;
    errno = 0;
    const long long r = strtoll(p, &e, 10);
    if (e == p || errno)
      return false;
    p = e;
    x = r;
    return true;
  }
  bool real(double &x) {
    skip_ws();
    if (p >= end)
      return false;
    char *e = nullptr;
    const double r = strtod(p, &e);
    if (e == p)
      return false;
    p = e;
    x = r;
    return true;
  }
};

std::string lower(std::string s) {
  for (auto &c : s)
    c = (char)tolower((unsigned char)c);
  return s;
}

int parse_ija(const std::string &buf, const char *path, Triplets &t) {
  Scan s{buf.data(), buf.data() + buf.size()};
  int64_t m, n, nnz;
  if (!s.int64(m) || !s.int64(n) || !s.int64(nnz) || m < 0 || n < 0 || nnz < 0) {
    set_error("Invalid IJA file header: %s", path);
    return KRANS_ERR_RUNTIME;
  }
  t.m = m;
  t.n = n;
  t.i.reserve((size_t)nnz);
  t.j.reserve((size_t)nnz);
  t.v.reserve((size_t)nnz);
  for (;;) {
    int64_t i, j;
    double v;
    const char *save = s.p;
    if (!s.int64(i) || !s.int64(j) || !s.real(v)) {
      s.p = save;
      break; // like `while (in >> i >> j >> value)`: stop at the first incomplete triplet
    }
    if (i < 0 || i >= m || j < 0 || j >= n) {
      set_error("IJA entry (%lld, %lld) outside a %lld x %lld matrix: %s", (long long)i, (long long)j,
                (long long)m, (long long)n, path);
      return KRANS_ERR_INVALID_ARGUMENT;
    }
    t.i.push_back(i);
    t.j.push_back(j);
    t.v.push_back(v);
  }
  if ((int64_t)t.v.size() != nnz)
    fprintf(stderr, "Warning: Expected %lld entries but read %zu\n", (long long)nnz, t.v.size());
  return KRANS_OK;
}

int parse_mtx(const std::string &buf, const char *path, Triplets &t) {
  const char *p = buf.data(), *end = p + buf.size();
  const char *nl = (const char *)memchr(p, '\n', (size_t)(end - p));
  const std::string head = lower(std::string(p, nl ? nl : end));
  char tag[64] = {0}, obj[64] = {0}, fmt[64] = {0}, field[64] = {0}, sym[64] = {0};
  if (sscanf(head.c_str(), "%63s %63s %63s %63s %63s", tag, obj, fmt, field, sym) != 5 ||
      strcmp(tag, "%%matrixmarket") != 0 || strcmp(obj, "matrix") != 0) {
    set_error("Failed to load Matrix Market file (bad banner): %s", path);
    return KRANS_ERR_RUNTIME;
  }
  if (strcmp(fmt, "coordinate") != 0) {
    set_error("Failed to load Matrix Market file (only coordinate format): %s", path);
    return KRANS_ERR_RUNTIME;
  }
  const bool pattern = strcmp(field, "pattern") == 0;
  if (!pattern && strcmp(field, "real") != 0 && strcmp(field, "integer") != 0 && strcmp(field, "double") != 0) {
    set_error("Failed to load Matrix Market file (field '%s' not supported): %s", field, path);
    return KRANS_ERR_RUNTIME;
  }
  const bool symm = strcmp(sym, "symmetric") == 0, skew = strcmp(sym, "skew-symmetric") == 0;
  if (!symm && !skew && strcmp(sym, "general") != 0) {
    set_error("Failed to load Matrix Market file (symmetry '%s' not supported): %s", sym, path);
    return KRANS_ERR_RUNTIME;
  }
  // skip the banner and comment lines
  p = nl ? nl + 1 : end;
  while (p < end) {
    const char *q = p;
    while (q < end && (*q == ' ' || *q == '\t'))
      q++;
    if (q < end && *q == '%') {
      const char *e = (const char *)memchr(q, '\n', (size_t)(end - q));
      p = e ? e + 1 : end;
      continue;
    }
    if (q < end && (*q == '\n' || *q == '\r')) {
      p = q + 1;
      continue;
    }
    break;
  }
  Scan s{p, end};
  int64_t m, n, nnz;
  if (!s.int64(m) || !s.int64(n) || !s.int64(nnz) || m < 0 || n < 0 || nnz < 0) {
    set_error("Failed to load Matrix Market file (bad size line): %s", path);
    return KRANS_ERR_RUNTIME;
  }
  t.m = m;
  t.n = n;
  const size_t cap = (size_t)nnz * ((symm || skew) ? 2 : 1);
  t.i.reserve(cap);
  t.j.reserve(cap);
  t.v.reserve(cap);
  for (int64_t k = 0; k < nnz; k++) {
    int64_t i, j;
    double v = 1.0;
    if (!s.int64(i) || !s.int64(j) || (!pattern && !s.real(v))) {
      set_error("Failed to load Matrix Market file (entry %lld of %lld): %s", (long long)(k + 1),
                (long long)nnz, path);
      return KRANS_ERR_RUNTIME;
    }
    i -= 1; // 1-based in the file
    j -= 1;
    if (i < 0 || i >= m || j < 0 || j >= n) {
      set_error("Matrix Market entry (%lld, %lld) outside a %lld x %lld matrix: %s", (long long)(i + 1),
                (long long)(j + 1), (long long)m, (long long)n, path);
      return KRANS_ERR_INVALID_ARGUMENT;
    }
    t.i.push_back(i);
    t.j.push_back(j);
    t.v.push_back(v);
    if ((symm || skew) && i != j) {
      t.i.push_back(j);
      t.j.push_back(i);
      t.v.push_back(skew ? -v : v);
    }
  }
  return KRANS_OK;
}

// CSR with columns ascending in each row; duplicates summed in file order
int to_csr(const Triplets &t, std::vector<int32_t> &rp, std::vector<int32_t> &ci, std::vector<double> &val) {
  if (t.m >= INT32_MAX || t.n >= INT32_MAX || (int64_t)t.v.size() >= INT32_MAX) {
    set_error("matrix too large for 32-bit CSR indices");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  const size_t z = t.v.size();
  std::vector<int64_t> cnt((size_t)t.m + 1, 0);
  for (size_t k = 0; k < z; k++)
    cnt[(size_t)t.i[k] + 1]++;
  for (int64_t r = 0; r < t.m; r++)
    cnt[(size_t)r + 1] += cnt[(size_t)r];
  std::vector<size_t> perm(z);
  {
    std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
    for (size_t k = 0; k < z; k++)
      perm[(size_t)pos[(size_t)t.i[k]]++] = k; // stable: file order within a row
  }
  rp.assign((size_t)t.m + 1, 0);
  ci.clear();
  val.clear();
  ci.reserve(z);
  val.reserve(z);
  std::vector<size_t> row;
  for (int64_t r = 0; r < t.m; r++) {
    row.assign(perm.begin() + cnt[(size_t)r], perm.begin() + cnt[(size_t)r + 1]);
    std::stable_sort(row.begin(), row.end(), [&](size_t a, size_t b) { return t.j[a] < t.j[b]; });
    for (size_t q = 0; q < row.size();) {
      const int64_t c = t.j[row[q]];
      double s = 0.0;
      for (; q < row.size() && t.j[row[q]] == c; q++)
        s += t.v[row[q]];
      ci.push_back((int32_t)c);
      val.push_back(s);
    }
    rp[(size_t)r + 1] = (int32_t)ci.size();
  }
  return KRANS_OK;
}

int read_any(const char *path, int format, std::vector<int32_t> &rp, std::vector<int32_t> &ci,
             std::vector<double> &val, int64_t *m, int64_t *n) {
  if (!path) {
    set_error("NULL path");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  if (format == KRANS_FMT_AUTO) {
    const char *dot = strrchr(path, '.');
    const std::string ext = dot ? lower(dot + 1) : "";
    if (ext == "mtx")
      format = KRANS_FMT_MTX;
    else if (ext == "ija")
      format = KRANS_FMT_IJA;
    else {
      set_error("Unsupported input format: expected .mtx or .ija (%s)", path);
      return KRANS_ERR_INVALID_ARGUMENT;
    }
  }
  if (format != KRANS_FMT_MTX && format != KRANS_FMT_IJA) {
    set_error("unknown matrix file format %d", format);
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  std::string buf;
  if (!read_file(path, buf)) {
    set_error("Cannot open file: %s", path);
    return KRANS_ERR_RUNTIME;
  }
  Triplets t;
  const int rc = format == KRANS_FMT_MTX ? parse_mtx(buf, path, t) : parse_ija(buf, path, t);
  if (rc != KRANS_OK)
    return rc;
  *m = t.m;
  *n = t.n;
  return to_csr(t, rp, ci, val);
}

} // namespace

extern "C" {

int krans_csr_read_host(const char *path, int format, int64_t *m, int64_t *n, int64_t *nnz, int32_t **row_ptr,
                        int32_t **col_idx, double **values) {
  if (!m || !n || !nnz || !row_ptr || !col_idx || !values) {
    set_error("krans_csr_read_host: NULL argument");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  *row_ptr = nullptr;
  *col_idx = nullptr;
  *values = nullptr;
  std::vector<int32_t> rp, ci;
  std::vector<double> val;
  const int rc = read_any(path, format, rp, ci, val, m, n);
  if (rc != KRANS_OK)
    return rc;
  *nnz = (int64_t)val.size();
  *row_ptr = (int32_t *)malloc(sizeof(int32_t) * rp.size());
  *col_idx = (int32_t *)malloc(sizeof(int32_t) * std::max<size_t>(ci.size(), 1));
  *values = (double *)malloc(sizeof(double) * std::max<size_t>(val.size(), 1));
  if (!*row_ptr || !*col_idx || !*values) {
    free(*row_ptr);
    free(*col_idx);
    free(*values);
    *row_ptr = nullptr;
    *col_idx = nullptr;
    *values = nullptr;
    set_error("krans_csr_read_host: out of host memory");
    return KRANS_ERR_OUT_OF_MEMORY;
  }
  std::copy(rp.begin(), rp.end(), *row_ptr);
  std::copy(ci.begin(), ci.end(), *col_idx);
  std::copy(val.begin(), val.end(), *values);
  return KRANS_OK;
}

void krans_host_free(void *p) { free(p); }

int krans_csr_load(krans_ctx *ctx, const char *path, int format, int flags, krans_mat **out) {
  if (!ctx || !out) {
    set_error("krans_csr_load: NULL argument");
    return KRANS_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  std::vector<int32_t> rp, ci;
  std::vector<double> val;
  int64_t m = 0, n = 0;
  const int rc = read_any(path, format, rp, ci, val, &m, &n);
  if (rc != KRANS_OK)
    return rc;
  return krans_csr_create(ctx, m, n, (int64_t)val.size(), rp.data(), ci.data(), val.data(), flags, out);
}

} // extern "C"
