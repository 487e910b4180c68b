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
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include "host_util.h"

namespace bcmg {

static thread_local std::string g_last_error;

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
  std::vector<int32_t> col(nz);
  std::vector<double> val(nz);
  for (size_t k = 0; k < nz; ++k) {
    int64_t p = pos[ci[k]]++;
    col[p] = cj[k];
    val[p] = cv[k];
  }
  // Sort each row by column (stable: duplicates keep file order) and merge.
  std::vector<int32_t> outrow(static_cast<size_t>(n) + 1, 0);
  std::vector<int32_t> perm;
  int64_t w = 0;
  std::vector<int32_t> ocol(nz);
  std::vector<double> oval(nz);
  for (int32_t i = 0; i < n; ++i) {
    int64_t b = cnt[i], e = cnt[i + 1];
    perm.resize(e - b);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int32_t x, int32_t y) {
      return col[b + x] < col[b + y];
    });
    int32_t last = -1;
    for (int32_t t : perm) {
      int32_t c = col[b + t];
      if (c == last) {
        oval[w - 1] += val[b + t];
      } else {
        ocol[w] = c;
        oval[w] = val[b + t];
        ++w;
        last = c;
      }
    }
    outrow[i + 1] = static_cast<int32_t>(w);
  }
  if (w > INT32_MAX)
    return set_error(BCMG_ERR_INVALID_MATRIX, "nnz %lld exceeds int32",
                     static_cast<long long>(w));
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
  std::memcpy(out->row, outrow.data(), sizeof(int32_t) * (n + 1));
  std::memcpy(out->col, ocol.data(), sizeof(int32_t) * w);
  std::memcpy(out->val, oval.data(), sizeof(double) * w);
  return BCMG_OK;
}

static void lower(char *s) {
  for (; *s; ++s)
    if (*s >= 'A' && *s <= 'Z') *s = static_cast<char>(*s - 'A' + 'a');
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
  std::vector<int32_t> ci, cj;
  std::vector<double> cv;
  size_t reserve = static_cast<size_t>(symmetric ? 2 * nz : nz);
  ci.reserve(reserve);
  cj.reserve(reserve);
  cv.reserve(reserve);
  for (long long k = 0; k < nz; ++k) {
    if (!fgets(line, sizeof(line), fp)) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': error reading record %lld of %lld", path,
                       k, nz);
    }
    long long i = 0, j = 0;
    double v = 1.0;
    int need = pattern ? 2 : 3;
    int r = pattern ? sscanf(line, "%lld %lld", &i, &j)
                    : sscanf(line, "%lld %lld %lf", &i, &j, &v);
    if (r != need) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': malformed record %lld", path, k);
    }
    ci.push_back(static_cast<int32_t>(i - 1));
    cj.push_back(static_cast<int32_t>(j - 1));
    cv.push_back(v);
    if (symmetric && i != j) {
      ci.push_back(static_cast<int32_t>(j - 1));
      cj.push_back(static_cast<int32_t>(i - 1));
      cv.push_back(v);
    }
  }
  fclose(fp);
  return coo_to_csr(static_cast<int32_t>(nr), static_cast<int32_t>(nc), ci, cj, cv,
                    out);
}

// Plain COO list reader (readMTX2Double, matrixIO.cu:194-289): "n nnz",
// then nnz 1-based row indices, nnz 1-based column indices, nnz values.
static bcmg_status read_coo_list(const char *path, bcmg_csr *out) {
  FILE *fp = fopen(path, "r");
  if (!fp) return set_error(BCMG_ERR_IO, "cannot open matrix file '%s'", path);
  long long n = 0, nz = 0;
  if (fscanf(fp, "%lld %lld", &n, &nz) != 2 || n <= 0 || nz < 0 || n > INT32_MAX) {
    fclose(fp);
    return set_error(BCMG_ERR_IO, "'%s': bad COO header", path);
  }
  std::vector<int32_t> ci(nz), cj(nz);
  std::vector<double> cv(nz);
  for (long long k = 0; k < nz; ++k) {
    long long t;
    if (fscanf(fp, "%lld", &t) != 1) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': short row list", path);
    }
    ci[k] = static_cast<int32_t>(t - 1);
  }
  for (long long k = 0; k < nz; ++k) {
    long long t;
    if (fscanf(fp, "%lld", &t) != 1) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': short column list", path);
    }
    cj[k] = static_cast<int32_t>(t - 1);
  }
  for (long long k = 0; k < nz; ++k) {
    if (fscanf(fp, "%lf", &cv[k]) != 1) {
      fclose(fp);
      return set_error(BCMG_ERR_IO, "'%s': short value list", path);
    }
  }
  fclose(fp);
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
  for (int32_t i = 0; i < A->n; ++i)
    for (int32_t j = A->row[i]; j < A->row[i + 1]; ++j)
      fprintf(fp, "%d   %d  %.18e\n", i + 1, A->col[j] + 1, A->val[j]);
  fclose(fp);
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
