// Matrix input/output, settings parsing and CSR validation (host code).
//
// Mirrors the reference's boundary:
//   readMatrixFromFile / readMTXDouble / readMTX2Double  src/matrix/matrixIO.cu:4-289
//   CSRMatrixPrintMM                                     src/matrix/matrixIO.cu:292-335
//   AMG::Params::initFromFile + checkP                   src/AMG/AMG.cu:8-18, 480-526
//   int_get_fp / double_get_fp                           src/AMG/utility.cu:7-25
// Differences, all deliberate: errors are returned instead of exit(); each
// row's columns are sorted and duplicates summed (the reference keeps file
// order although _makeAH_warp assumes sorted rows with a diagonal).
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "host_util.h"

namespace bcmg {

static thread_local std::string g_last_error;

// Threads for reading or writing `bytes` of matrix text: one per 4 MB, at
// most the hardware's threads and 16.
static int io_threads(size_t bytes) {
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  return static_cast<int>(std::min<size_t>({bytes / (size_t{4} << 20) + 1, hw, 16}));
}

// Runs f(t) for t = 0 .. T-1, t = 0 on the calling thread (a thread that
// cannot be started runs its share on the caller too).
template <typename F>
static void run_threads(int T, const F &f) {
  std::vector<std::thread> pool;
  int started = 1;
  try {
    for (; started < T; ++started) pool.emplace_back(f, started);
  } catch (...) {
  }
  for (int t = started; t < T; ++t) f(t);
  f(0);
  for (auto &th : pool) th.join();
}

bcmg_status set_error(bcmg_status code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

const char *last_error() { return g_last_error.c_str(); }

// Builds a CSR with sorted columns and summed duplicates from COO triplets.
// Row/column indices are 0-based and must be in range.
static bcmg_status coo_to_csr(int32_t n, int32_t m, std::vector<int32_t> &ci,
                              std::vector<int32_t> &cj, std::vector<double> &cv,
                              bcmg_csr *out) {
  const size_t nz = ci.size();
  for (size_t k = 0; k < nz; ++k) {
    if (ci[k] < 0 || ci[k] >= n || cj[k] < 0 || cj[k] >= m)
      return set_error(BCMG_ERR_INVALID_MATRIX,
                       "entry %zu has index (%d, %d) outside %d x %d", k,
                       ci[k] + 1, cj[k] + 1, n, m);
  }
  std::vector<int64_t> cnt(static_cast<size_t>(n) + 1, 0);
  for (size_t k = 0; k < nz; ++k) cnt[ci[k] + 1]++;
  for (int32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
  // Scatter into rows (file order within a row), then per row: a row whose
  // columns already increase strictly is kept as it is; otherwise it is
  // sorted by column (stable: duplicates keep file order) and duplicates are
  // summed, in place.  Rows in parallel.
  std::unique_ptr<int32_t[]> col(new int32_t[nz > 0 ? nz : 1]);
  std::unique_ptr<double[]> val(new double[nz > 0 ? nz : 1]);
  for (size_t k = 0; k < nz; ++k) {
    int64_t p = pos[ci[k]]++;
    col[p] = cj[k];
    val[p] = cv[k];
  }
  const int T = io_threads(nz * 16);
  std::vector<int64_t> unique(static_cast<size_t>(n), 0);
  run_threads(T, [&](int t) {
    const int32_t i0 = static_cast<int32_t>(static_cast<int64_t>(n) * t / T);
    const int32_t i1 = static_cast<int32_t>(static_cast<int64_t>(n) * (t + 1) / T);
    std::vector<int32_t> perm, tcol;
    std::vector<double> tval;
    for (int32_t i = i0; i < i1; ++i) {
      const int64_t b = cnt[i], e = cnt[i + 1];
      bool increasing = true;
      for (int64_t k = b + 1; k < e && increasing; ++k) increasing = col[k - 1] < col[k];
      if (increasing) {
        unique[i] = e - b;
        continue;
      }
      perm.resize(e - b);
      std::iota(perm.begin(), perm.end(), 0);
      std::stable_sort(perm.begin(), perm.end(), [&](int32_t x, int32_t y) {
        return col[b + x] < col[b + y];
      });
      tcol.clear();
      tval.clear();
      for (int32_t q : perm) {
        const int32_t c = col[b + q];
        if (!tcol.empty() && tcol.back() == c) {
          tval.back() += val[b + q];
        } else {
          tcol.push_back(c);
          tval.push_back(val[b + q]);
        }
      }
      std::copy(tcol.begin(), tcol.end(), col.get() + b);
      std::copy(tval.begin(), tval.end(), val.get() + b);
      unique[i] = static_cast<int64_t>(tcol.size());
    }
  });
  int64_t w = 0;
  for (int32_t i = 0; i < n; ++i) {
    w += unique[i];
    if (w > INT32_MAX)
      return set_error(BCMG_ERR_INVALID_MATRIX, "nnz %lld exceeds int32",
                       static_cast<long long>(w));
  }
  out->n = n;
  out->m = m;
  out->nnz = static_cast<int32_t>(w);
  out->row = static_cast<int32_t *>(malloc(sizeof(int32_t) * (n + 1)));
  out->col = static_cast<int32_t *>(malloc(sizeof(int32_t) * (w > 0 ? w : 1)));
  out->val = static_cast<double *>(malloc(sizeof(double) * (w > 0 ? w : 1)));
  if (!out->row || !out->col || !out->val) {
    free(out->row);
    free(out->col);
    free(out->val);
    out->row = nullptr;
    out->col = nullptr;
    out->val = nullptr;
    return set_error(BCMG_ERR_ALLOC, "host allocation of CSR failed");
  }
  out->row[0] = 0;
  for (int32_t i = 0; i < n; ++i) out->row[i + 1] = out->row[i] + static_cast<int32_t>(unique[i]);
  run_threads(T, [&](int t) {
    const int32_t i0 = static_cast<int32_t>(static_cast<int64_t>(n) * t / T);
    const int32_t i1 = static_cast<int32_t>(static_cast<int64_t>(n) * (t + 1) / T);
    for (int32_t i = i0; i < i1; ++i) {
      std::copy(col.get() + cnt[i], col.get() + cnt[i] + unique[i], out->col + out->row[i]);
      std::copy(val.get() + cnt[i], val.get() + cnt[i] + unique[i], out->val + out->row[i]);
    }
  });
  return BCMG_OK;
}

static void lower(char *s) {
  for (; *s; ++s)
    if (*s >= 'A' && *s <= 'Z') *s = static_cast<char>(*s - 'A' + 'a');
}

static inline bool mm_space(char c) {
  return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

// One integer as %lld reads it: leading white space, an optional sign, at
// least one digit (saturating on overflow); nullptr if there is none.
static const char *scan_ll(const char *p, const char *e, long long *out) {
  while (p < e && mm_space(*p)) ++p;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
  if (p >= e || *p < '0' || *p > '9') return nullptr;
  unsigned long long v = 0;
  for (; p < e && *p >= '0' && *p <= '9'; ++p)
    v = v > (ULLONG_MAX - 9) / 10 ? ULLONG_MAX : v * 10 + static_cast<unsigned>(*p - '0');
  v = std::min(v, static_cast<unsigned long long>(LLONG_MAX));
  *out = neg ? -static_cast<long long>(v) : static_cast<long long>(v);
  return p;
}

// One number as %lf reads it (strtod's syntax): std::from_chars for the
// usual forms, strtod where from_chars stops short of what strtod would
// take (a hexadecimal float, a value out of range).  The text is
// NUL-terminated, so strtod stays inside it.
static const char *scan_double(const char *p, const char *e, double *out) {
  while (p < e && mm_space(*p)) ++p;
  if (p >= e) return nullptr;
  const char *q = p;
  if (*q == '+') {  // from_chars takes no plus sign
    ++q;
    if (q < e && (*q == '+' || *q == '-')) return nullptr;
  }
  double v = 0.0;
  const auto r = std::from_chars(q, e, v);
  const bool more = r.ptr < e && (std::isalnum(static_cast<unsigned char>(*r.ptr)) || *r.ptr == '.');
  if (r.ec == std::errc() && !more) {
    *out = v;
    return r.ptr;
  }
  char *end = nullptr;
  const double s = std::strtod(p, &end);
  if (end == p) return nullptr;
  *out = s;
  return end;
}

// The first nz lines of `text` as Matrix-Market records "i j [v]" (1-based;
// v = 1 for a pattern matrix), in file order, with the mirrored entry of an
// off-diagonal record right after it for symmetric storage.  The text is cut
// into line-aligned chunks parsed by threads.  *bad = the first malformed
// record (-1: none); *lines = the lines the text has (fewer than nz: records
// are missing).
static void parse_records(const std::string &text, long long nz, bool pattern, bool symmetric,
                          std::vector<int32_t> &ci, std::vector<int32_t> &cj,
                          std::vector<double> &cv, long long *bad, long long *lines) {
  const char *base = text.c_str();
  const size_t size = text.size();
  const int T = io_threads(size);
  std::vector<size_t> cut(T + 1, size);
  cut[0] = 0;
  for (int t = 1; t < T; ++t) {
    size_t c = std::max(cut[t - 1], size * static_cast<size_t>(t) / T);
    while (c > 0 && c < size && base[c - 1] != '\n') ++c;
    cut[t] = c;
  }
  // Lines per chunk (every chunk but the last ends just after a newline).
  std::vector<long long> count(T, 0), first(T + 1, 0), tbad(T, -1);
  run_threads(T, [&](int t) {
    const char *p = base + cut[t], *e = base + cut[t + 1];
    long long c = std::count(p, e, '\n');
    if (e > p && e[-1] != '\n') ++c;
    count[t] = c;
  });
  for (int t = 0; t < T; ++t) first[t + 1] = first[t] + count[t];
  *lines = first[T];
  // Every chunk writes its entries from `per` slots per record before it
  // (one record gives at most `per` entries); a symmetric file's entries
  // are compacted afterwards, chunk by chunk in file order.
  const size_t per = symmetric ? 2 : 1;
  const size_t records = static_cast<size_t>(std::min(first[T], nz));
  ci.resize(records * per);
  cj.resize(records * per);
  cv.resize(records * per);
  std::vector<size_t> made(T, 0);
  run_threads(T, [&](int t) {
    long long g = first[t];
    if (g >= nz) return;
    const long long mine = std::min(count[t], nz - g);
    size_t w = static_cast<size_t>(g) * per;
    const size_t w0 = w;
    const char *p = base + cut[t], *end = base + cut[t + 1];
    for (long long k = 0; k < mine; ++k, ++g) {
      const char *nl = static_cast<const char *>(std::memchr(p, '\n', end - p));
      const char *le = nl ? nl : end;
      long long i = 0, j = 0;
      double v = 1.0;
      const char *q = scan_ll(p, le, &i);
      if (q) q = scan_ll(q, le, &j);
      if (q && !pattern) q = scan_double(q, le, &v);
      if (!q) {
        tbad[t] = g;
        return;
      }
      ci[w] = static_cast<int32_t>(i - 1);
      cj[w] = static_cast<int32_t>(j - 1);
      cv[w++] = v;
      if (symmetric && i != j) {
        ci[w] = static_cast<int32_t>(j - 1);
        cj[w] = static_cast<int32_t>(i - 1);
        cv[w++] = v;
      }
      p = nl ? nl + 1 : end;
    }
    made[t] = w - w0;
  });
  *bad = -1;
  for (int t = 0; t < T; ++t)
    if (tbad[t] >= 0) {
      *bad = tbad[t];  // chunks are in file order: the first one found is the first
      return;
    }
  if (per == 1) return;  // one entry per record: already in place
  size_t at = 0;
  for (int t = 0; t < T && first[t] < nz; ++t) {
    const size_t from = static_cast<size_t>(first[t]) * per;
    if (at != from) {
      std::memmove(ci.data() + at, ci.data() + from, made[t] * sizeof(int32_t));
      std::memmove(cj.data() + at, cj.data() + from, made[t] * sizeof(int32_t));
      std::memmove(cv.data() + at, cv.data() + from, made[t] * sizeof(double));
    }
    at += made[t];
  }
  ci.resize(at);
  cj.resize(at);
  cv.resize(at);
}

// Matrix Market coordinate reader (readMTXDouble, matrixIO.cu:33-192):
// real/integer/pattern values, general or symmetric storage (symmetric is
// mirrored off the diagonal, matrixIO.cu:106-133).
static bcmg_status read_mm(const char *path, bcmg_csr *out) {
  FILE *fp = fopen(path, "r");
  if (!fp) return set_error(BCMG_ERR_IO, "cannot open matrix file '%s'", path);
  char line[4096];
  if (!fgets(line, sizeof(line), fp)) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': empty file", path);
  }
  char banner[64] = {0}, obj[64] = {0}, fmt[64] = {0}, field[64] = {0},
       sym[64] = {0};
  int got = sscanf(line, "%63s %63s %63s %63s %63s", banner, obj, fmt, field, sym);
  lower(obj);
  lower(fmt);
  lower(field);
  lower(sym);
  if (got < 5 || std::strcmp(banner, "%%MatrixMarket") != 0 ||
      std::strcmp(obj, "matrix") != 0 || std::strcmp(fmt, "coordinate") != 0) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': not a MatrixMarket coordinate matrix", path);
  }
  const bool pattern = std::strcmp(field, "pattern") == 0;
  if (!pattern && std::strcmp(field, "real") != 0 &&
      std::strcmp(field, "integer") != 0 && std::strcmp(field, "double") != 0) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': only real matrices are read, not '%s'",
                     path, field);
  }
  bool symmetric = false;
  if (std::strcmp(sym, "symmetric") == 0) {
    symmetric = true;
  } else if (std::strcmp(sym, "general") != 0) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': unhandled storage scheme '%s'", path, sym);
  }
  // Skip comments (matrixIO.cu:61-62).
  do {
    if (!fgets(line, sizeof(line), fp)) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': missing size line", path);
    }
  } while (line[0] == '%');
  long long nr = 0, nc = 0, nz = 0;
  if (sscanf(line, "%lld %lld %lld", &nr, &nc, &nz) != 3 || nr <= 0 || nc <= 0 ||
      nz < 0 || nr > INT32_MAX || nc > INT32_MAX) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': bad size line", path);
  }
  // The records: the rest of the file in one read, one record per line.
  std::string body;
  {
    const long here = ftell(fp);
    if (here >= 0 && fseek(fp, 0, SEEK_END) == 0) {
      const long end = ftell(fp);
      if (end > here) body.reserve(static_cast<size_t>(end - here));
      fseek(fp, here, SEEK_SET);
    }
    char chunk[1 << 16];
    size_t got_bytes;
    while ((got_bytes = fread(chunk, 1, sizeof(chunk), fp)) > 0) body.append(chunk, got_bytes);
    const bool failed = ferror(fp) != 0;
    fclose(fp);
    if (failed) return set_error(BCMG_ERR_IO, "'%s': read error", path);
  }
  std::vector<int32_t> ci, cj;
  std::vector<double> cv;
  long long bad = -1, lines = 0;
  parse_records(body, nz, pattern, symmetric, ci, cj, cv, &bad, &lines);
  std::string().swap(body);
  if (bad >= 0) return set_error(BCMG_ERR_IO, "'%s': malformed record %lld", path, bad);
  if (lines < nz)
    return set_error(BCMG_ERR_IO, "'%s': error reading record %lld of %lld", path, lines,
                     nz);
  return coo_to_csr(static_cast<int32_t>(nr), static_cast<int32_t>(nc), ci, cj, cv,
                    out);
}

// Plain COO list reader (readMTX2Double, matrixIO.cu:194-289): "n nnz",
// then nnz 1-based row indices, nnz 1-based column indices, nnz values.
static bcmg_status read_coo_list(const char *path, bcmg_csr *out) {
  FILE *fp = fopen(path, "r");
  if (!fp) return set_error(BCMG_ERR_IO, "cannot open matrix file '%s'", path);
  std::string text;
  {
    if (fseek(fp, 0, SEEK_END) == 0) {
      const long end = ftell(fp);
      if (end > 0) text.reserve(static_cast<size_t>(end));
      fseek(fp, 0, SEEK_SET);
    }
    char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), fp)) > 0) text.append(chunk, got);
    const bool failed = ferror(fp) != 0;
    fclose(fp);
    if (failed) return set_error(BCMG_ERR_IO, "'%s': read error", path);
  }
  // Numbers read one after the other, each from where the previous one
  // stopped, as fscanf("%lld") / fscanf("%lf") on the stream read them.
  const char *p = text.c_str(), *e = p + text.size();
  long long n = 0, nz = 0;
  p = scan_ll(p, e, &n);
  if (p) p = scan_ll(p, e, &nz);
  if (!p || n <= 0 || nz < 0 || n > INT32_MAX)
    return set_error(BCMG_ERR_IO, "'%s': bad COO header", path);
  // A number takes at least two bytes, so no list is longer than this.
  const size_t cap = std::min(static_cast<size_t>(nz), text.size() / 2 + 1);
  std::vector<int32_t> ci, cj;
  std::vector<double> cv;
  ci.reserve(cap);
  cj.reserve(cap);
  cv.reserve(cap);
  for (long long k = 0; k < nz; ++k) {
    long long t = 0;
    if (!(p = scan_ll(p, e, &t))) return set_error(BCMG_ERR_IO, "'%s': short row list", path);
    ci.push_back(static_cast<int32_t>(t - 1));
  }
  for (long long k = 0; k < nz; ++k) {
    long long t = 0;
    if (!(p = scan_ll(p, e, &t)))
      return set_error(BCMG_ERR_IO, "'%s': short column list", path);
    cj.push_back(static_cast<int32_t>(t - 1));
  }
  for (long long k = 0; k < nz; ++k) {
    double v = 0.0;
    if (!(p = scan_double(p, e, &v)))
      return set_error(BCMG_ERR_IO, "'%s': short value list", path);
    cv.push_back(v);
  }
  std::string().swap(text);
  return coo_to_csr(static_cast<int32_t>(n), static_cast<int32_t>(n), ci, cj, cv,
                    out);
}

// One "value % comment" settings line (int_get_fp / double_get_fp,
// src/AMG/utility.cu:7-25): the text before the first '%' is parsed.
static bool settings_line(FILE *fp, char *buf, size_t cap) {
  if (!fgets(buf, static_cast<int>(cap), fp)) return false;
  char *pct = std::strchr(buf, '%');
  if (pct) *pct = '\0';
  return true;
}

static bool parse_int(const char *s, int *v) {
  char *end = nullptr;
  errno = 0;
  long x = std::strtol(s, &end, 10);
  if (end == s || errno != 0 || x < INT32_MIN || x > INT32_MAX) return false;
  *v = static_cast<int>(x);
  return true;
}

static bool parse_double(const char *s, double *v) {
  char *end = nullptr;
  errno = 0;
  double x = std::strtod(s, &end);
  if (end == s || errno != 0) return false;
  *v = x;
  return true;
}

}  // namespace bcmg

using namespace bcmg;

extern "C" {

const char *bcmg_last_error(void) { return bcmg::last_error(); }

const char *bcmg_status_string(int status) {
  switch (status) {
    case BCMG_OK: return "BCMG_OK";
    case BCMG_ERR_PARAM: return "BCMG_ERR_PARAM";
    case BCMG_ERR_IO: return "BCMG_ERR_IO";
    case BCMG_ERR_ALLOC: return "BCMG_ERR_ALLOC";
    case BCMG_ERR_CUDA: return "BCMG_ERR_CUDA";
    case BCMG_ERR_INDEFINITE: return "BCMG_ERR_INDEFINITE";
    case BCMG_ERR_NOT_CONVERGED: return "BCMG_ERR_NOT_CONVERGED";
    case BCMG_ERR_DEVICE_TIMEOUT: return "BCMG_ERR_DEVICE_TIMEOUT";
    case BCMG_ERR_INVALID_MATRIX: return "BCMG_ERR_INVALID_MATRIX";
    case BCMG_ERR_UNSUPPORTED: return "BCMG_ERR_UNSUPPORTED";
    case BCMG_ERR_INTERNAL: return "BCMG_ERR_INTERNAL";
    case BCMG_ERR_PENDING: return "BCMG_ERR_PENDING";
    default: return "BCMG_ERR_UNKNOWN";
  }
}

const char *bcmg_version(void) { return "bcmg-b200 0.1 (sm_100a)"; }

bcmg_status bcmg_read_matrix(const char *path, int m_type, bcmg_csr *out) {
  if (!path || !out) return set_error(BCMG_ERR_PARAM, "null argument");
  std::memset(out, 0, sizeof(*out));
  if (m_type == 0) return read_mm(path, out);
  if (m_type == 1) return read_coo_list(path, out);
  return set_error(BCMG_ERR_PARAM, "unknown matrix file type %d (0 MM, 1 COO)",
                   m_type);
}

bcmg_status bcmg_write_matrix_mm(const char *path, const bcmg_csr *A) {
  if (!path || !A) return set_error(BCMG_ERR_PARAM, "null argument");
  FILE *fp = fopen(path, "w");
  if (!fp) return set_error(BCMG_ERR_IO, "cannot write '%s'", path);
  fprintf(fp, "%%%%MatrixMarket matrix coordinate real general\n");
  fprintf(fp, "%d  %d %d \n", A->n, A->m, A->nnz);
  // Rows formatted in parallel (ranges of rows, each into its own text),
  // written in order: the same bytes as one fprintf per entry.
  const int T = io_threads(static_cast<size_t>(std::max(A->nnz, 0)) * 48);
  std::vector<std::string> text(T);
  run_threads(T, [&](int t) {
    const int32_t i0 = static_cast<int32_t>(static_cast<int64_t>(A->n) * t / T);
    const int32_t i1 = static_cast<int32_t>(static_cast<int64_t>(A->n) * (t + 1) / T);
    std::string &s = text[t];
    s.reserve(static_cast<size_t>(A->row[i1] - A->row[i0]) * 48);
    char rec[96];
    for (int32_t i = i0; i < i1; ++i)
      for (int32_t j = A->row[i]; j < A->row[i + 1]; ++j) {
        const int len =
            snprintf(rec, sizeof(rec), "%d   %d  %.18e\n", i + 1, A->col[j] + 1, A->val[j]);
        s.append(rec, static_cast<size_t>(std::min<int>(len, sizeof(rec) - 1)));
      }
  });
  bool ok = true;
  for (const std::string &s : text)
    ok = ok && fwrite(s.data(), 1, s.size(), fp) == s.size();
  ok = (fclose(fp) == 0) && ok;
  if (!ok) return set_error(BCMG_ERR_IO, "error writing '%s'", path);
  return BCMG_OK;
}

void bcmg_csr_free(bcmg_csr *A) {
  if (!A) return;
  free(A->row);
  free(A->col);
  free(A->val);
  A->row = nullptr;
  A->col = nullptr;
  A->val = nullptr;
  A->n = A->m = A->nnz = 0;
}

bcmg_status bcmg_csr_check(const bcmg_csr *A) {
  if (!A || !A->row || (A->nnz > 0 && (!A->col || !A->val)))
    return set_error(BCMG_ERR_PARAM, "null CSR array");
  if (A->n <= 0 || A->n != A->m)
    return set_error(BCMG_ERR_INVALID_MATRIX, "matrix must be square with n > 0 (%d x %d)",
                     A->n, A->m);
  if (A->row[0] != 0 || A->row[A->n] != A->nnz)
    return set_error(BCMG_ERR_INVALID_MATRIX, "row pointer does not span [0, nnz]");
  for (int32_t i = 0; i < A->n; ++i) {
    int32_t b = A->row[i], e = A->row[i + 1];
    if (e < b) return set_error(BCMG_ERR_INVALID_MATRIX, "row %d has negative length", i);
    bool diag = false;
    for (int32_t j = b; j < e; ++j) {
      int32_t c = A->col[j];
      if (c < 0 || c >= A->m)
        return set_error(BCMG_ERR_INVALID_MATRIX, "row %d: column %d out of range", i, c);
      if (j > b && A->col[j - 1] >= c)
        return set_error(BCMG_ERR_INVALID_MATRIX,
                         "row %d: columns not strictly increasing at position %d", i,
                         j - b);
      if (!std::isfinite(A->val[j]))
        return set_error(BCMG_ERR_INVALID_MATRIX, "row %d: non-finite value", i);
      if (c == i) diag = true;
    }
    if (!diag)
      return set_error(BCMG_ERR_INVALID_MATRIX,
                       "row %d has no diagonal entry (the AH builder needs one)", i);
  }
  return BCMG_OK;
}

// AMGsettings_base:1-14.
void bcmg_params_default(bcmg_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->solver_type = 0;
  p->max_hrc = 1;
  p->conv_ratio = 0.8;
  p->matchtype = 3;
  p->aggrsweeps = 2;
  p->aggrtype = 0;
  p->max_levels = 39;
  p->cycle_type = 0;
  p->coarse_solver = 4;
  p->relax_type = 4;
  p->relaxnumber_coarse = 20;
  p->prerelax_sweeps = 1;
  p->postrelax_sweeps = 1;
  p->itnlim = 200000;
  p->rtol = 1.e-6;
}

// checkP (AMG.cu:8-18) applied as in initFromFile (AMG.cu:492-516), plus
// range checks the reference does not make (they would crash it later).
bcmg_status bcmg_params_check(const bcmg_params *p) {
  if (!p) return set_error(BCMG_ERR_PARAM, "null params");
  if (p->solver_type < 0 || p->solver_type > 2)
    return set_error(BCMG_ERR_PARAM, "No parameter %d for solver_type", p->solver_type);
  if (p->aggrtype != 0 && p->aggrtype != 1)
    return set_error(BCMG_ERR_PARAM, "No parameter %d for aggrtype", p->aggrtype);
  // 3 = K-cycle: the reference carries the code (GAMG_cycle.cu:88-100) but its
  // checkP rejects the value (AMG.cu:508); it is accepted here.
  if (p->cycle_type < 0 || p->cycle_type > 3)
    return set_error(BCMG_ERR_PARAM, "No parameter %d for cycle_type", p->cycle_type);
  if (p->coarse_solver != 0 && p->coarse_solver != 4)
    return set_error(BCMG_ERR_PARAM, "No parameter %d for coarse_solver", p->coarse_solver);
  if (p->relax_type != 0 && p->relax_type != 4)
    return set_error(BCMG_ERR_PARAM, "No parameter %d for relax_type", p->relax_type);
  if (p->max_hrc < 1) return set_error(BCMG_ERR_PARAM, "max_hrc must be >= 1");
  if (p->aggrsweeps < 1) return set_error(BCMG_ERR_PARAM, "aggrsweeps must be >= 1");
  if (p->max_levels < 1) return set_error(BCMG_ERR_PARAM, "max_levels must be >= 1");
  if (p->prerelax_sweeps < 0 || p->postrelax_sweeps < 0 || p->relaxnumber_coarse < 0)
    return set_error(BCMG_ERR_PARAM, "sweep counts must be >= 0");
  if (p->itnlim < 1) return set_error(BCMG_ERR_PARAM, "itnlim must be >= 1");
  if (!(p->rtol >= 0.0)) return set_error(BCMG_ERR_PARAM, "rtol must be >= 0");
  return BCMG_OK;
}

// Settings file in the reference's line order (AMG.cu:491-522):
// solver_type, max_hrc, conv_ratio, aggrsweeps, aggrtype, max_levels,
// cycle_type, coarse_solver, relax_type, relaxnumber_coarse, prerelax,
// postrelax, itnlim, rtol; matchtype is forced to 3 (AMG.cu:497).
bcmg_status bcmg_params_from_file(const char *path, bcmg_params *p) {
  if (!path || !p) return set_error(BCMG_ERR_PARAM, "null argument");
  FILE *fp = fopen(path, "r");
  if (!fp) return set_error(BCMG_ERR_IO, "Setting file not found: '%s'", path);
  char buf[1025];
  bcmg_params q;
  std::memset(&q, 0, sizeof(q));
  struct Field {
    const char *name;
    int *ip;
    double *dp;
  } fields[] = {{"solver_type", &q.solver_type, nullptr},
                {"max_hrc", &q.max_hrc, nullptr},
                {"conv_ratio", nullptr, &q.conv_ratio},
                {"aggrsweeps", &q.aggrsweeps, nullptr},
                {"aggrtype", &q.aggrtype, nullptr},
                {"max_levels", &q.max_levels, nullptr},
                {"cycle_type", &q.cycle_type, nullptr},
                {"coarse_solver", &q.coarse_solver, nullptr},
                {"relax_type", &q.relax_type, nullptr},
                {"relaxnumber_coarse", &q.relaxnumber_coarse, nullptr},
                {"prerelax_sweeps", &q.prerelax_sweeps, nullptr},
                {"postrelax_sweeps", &q.postrelax_sweeps, nullptr},
                {"itnlim", &q.itnlim, nullptr},
                {"rtol", nullptr, &q.rtol}};
  for (const Field &f : fields) {
    if (!settings_line(fp, buf, sizeof(buf))) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': missing line for %s", path, f.name);
    }
    bool ok = f.ip ? parse_int(buf, f.ip) : parse_double(buf, f.dp);
    if (!ok) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': cannot parse %s from '%s'", path, f.name, buf);
    }
  }
  fclose(fp);
  q.matchtype = 3;
  BCMG_TRY(bcmg_params_check(&q));
  *p = q;
  return BCMG_OK;
}

void bcmg_ext_default(bcmg_ext *e) {
  std::memset(e, 0, sizeof(*e));
  e->precision = BCMG_PREC_FP64;
  e->coarse_storage = BCMG_STORE_FP32;
  e->replace_every = 0;
  e->use_graphs = 1;
  e->device = 0;
  e->verbose = 0;
  e->max_device_seconds = 2.0;
  e->stream = nullptr;
  e->sliced = 1;
  e->autotune = 1;
  e->narrow_values = 1;
  e->match_step_limit = 0;
}

}  // extern "C"
