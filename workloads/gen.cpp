// Deterministic synthetic inputs for the solve path (host code): the
// workload generators shared by the tests, bench.py's GPU arm and its CPU
// baseline.  Built as its own library (libworkloads.so) so that neither the
// product library nor the CPU oracle carries them.
//
// The reference ships no test matrices (its only sample, pi8grid6.mtx, is
// absent), so every workload is generated here from fixed seeds with one
// generator family: splitmix64 for uniforms, Box-Muller for normals.
// Matrices come out canonical: sorted columns, explicit diagonal, 0-based,
// rows in x-fastest lexicographic order for grids.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {
/* Same layout as bcmg_csr: 0-based CSR, int32 indices, FP64 values. */
typedef struct {
  int32_t n, m, nnz;
  int32_t *row;
  int32_t *col;
  double *val;
} wl_csr;
}

namespace wl {
namespace {

enum { WL_OK = 0, WL_ERR_PARAM = 1, WL_ERR_ALLOC = 3 };

thread_local char g_err[256];

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define WL_TRY(expr)           \
  do {                         \
    int _st = (expr);          \
    if (_st != WL_OK) return _st; \
  } while (0)

void csr_free(wl_csr *c) {
  if (!c) return;
  std::free(c->row);
  std::free(c->col);
  std::free(c->val);
  c->row = c->col = nullptr;
  c->val = nullptr;
}

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
  }
  // Uniform in [0, 1) with 53 random bits.
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
};

// Standard normals by Box-Muller, consumed in pairs.
struct Normal {
  SplitMix64 rng;
  bool have = false;
  double spare = 0.0;
  explicit Normal(uint64_t seed) : rng(seed) {}
  double next() {
    if (have) {
      have = false;
      return spare;
    }
    double u1 = 1.0 - rng.uniform();  // (0, 1]
    double u2 = rng.uniform();
    double r = std::sqrt(-2.0 * std::log(u1));
    double t = 6.283185307179586476925286766559 * u2;
    spare = r * std::sin(t);
    have = true;
    return r * std::cos(t);
  }
};

int alloc_csr(int32_t n, int64_t nnz, wl_csr *out) {
  if (nnz > INT32_MAX) return set_error(WL_ERR_PARAM, "nnz %lld exceeds int32", (long long)nnz);
  out->n = out->m = n;
  out->nnz = static_cast<int32_t>(nnz);
  out->row = static_cast<int32_t *>(malloc(sizeof(int32_t) * (n + 1)));
  out->col = static_cast<int32_t *>(malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1)));
  out->val = static_cast<double *>(malloc(sizeof(double) * (nnz > 0 ? nnz : 1)));
  if (!out->row || !out->col || !out->val) {
    csr_free(out);
    return set_error(WL_ERR_ALLOC, "host allocation failed");
  }
  return WL_OK;
}

}  // namespace
}  // namespace wl

using namespace wl;

extern "C" {

const char *wl_last_error(void) { return g_err; }

void wl_csr_free(wl_csr *c) { csr_free(c); }

int wl_poisson(int stencil, int32_t nx, int32_t ny, int32_t nz, wl_csr *out) {
  if (!out) return set_error(WL_ERR_PARAM, "null output");
  std::memset(out, 0, sizeof(*out));
  if (stencil == 5) nz = 1;
  if (nx <= 0 || ny <= 0 || nz <= 0)
    return set_error(WL_ERR_PARAM, "grid sizes must be positive");
  if (stencil != 5 && stencil != 7 && stencil != 27)
    return set_error(WL_ERR_PARAM, "stencil must be 5, 7 or 27");
  const int64_t n64 = static_cast<int64_t>(nx) * ny * nz;
  if (n64 > INT32_MAX) return set_error(WL_ERR_PARAM, "grid too large for int32");
  const int32_t n = static_cast<int32_t>(n64);
  // Offsets in increasing linear-index order so rows come out sorted.
  std::vector<int> ox, oy, oz;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int manh = std::abs(dx) + std::abs(dy) + std::abs(dz);
        bool take = false;
        if (stencil == 27) take = true;
        if (stencil == 7) take = manh <= 1;
        if (stencil == 5) take = dz == 0 && manh <= 1;
        if (take) {
          ox.push_back(dx);
          oy.push_back(dy);
          oz.push_back(dz);
        }
      }
  const double diag = stencil == 27 ? 26.0 : (stencil == 7 ? 6.0 : 4.0);
  int64_t cap = static_cast<int64_t>(n) * static_cast<int64_t>(ox.size());
  std::vector<int32_t> col;
  std::vector<double> val;
  col.reserve(cap);
  val.reserve(cap);
  std::vector<int32_t> row(static_cast<size_t>(n) + 1, 0);
  int32_t r = 0;
  for (int32_t z = 0; z < nz; ++z)
    for (int32_t y = 0; y < ny; ++y)
      for (int32_t x = 0; x < nx; ++x, ++r) {
        for (size_t k = 0; k < ox.size(); ++k) {
          int32_t xx = x + ox[k], yy = y + oy[k], zz = z + oz[k];
          if (xx < 0 || yy < 0 || zz < 0 || xx >= nx || yy >= ny || zz >= nz) continue;
          int32_t c = (zz * ny + yy) * nx + xx;
          col.push_back(c);
          val.push_back(c == r ? diag : -1.0);
        }
        row[r + 1] = static_cast<int32_t>(col.size());
      }
  WL_TRY(alloc_csr(n, static_cast<int64_t>(col.size()), out));
  std::memcpy(out->row, row.data(), sizeof(int32_t) * (n + 1));
  std::memcpy(out->col, col.data(), sizeof(int32_t) * col.size());
  std::memcpy(out->val, val.data(), sizeof(double) * val.size());
  return WL_OK;
}

int wl_fv2d(int32_t nx, int32_t ny, uint64_t seed, double aniso, wl_csr *out) {
  if (!out) return set_error(WL_ERR_PARAM, "null output");
  std::memset(out, 0, sizeof(*out));
  if (nx <= 0 || ny <= 0) return set_error(WL_ERR_PARAM, "grid sizes must be positive");
  const int64_t n64 = static_cast<int64_t>(nx) * ny;
  if (n64 * 5 > INT32_MAX) return set_error(WL_ERR_PARAM, "grid too large");
  const int32_t n = static_cast<int32_t>(n64);
  std::vector<double> g0(n), g(n), K(n);
  Normal nrm(seed);
  for (int32_t c = 0; c < n; ++c) g0[c] = nrm.next();
  for (int32_t y = 0; y < ny; ++y)
    for (int32_t x = 0; x < nx; ++x) {
      double s = 0.0;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int32_t xx = std::min(std::max(x + dx, 0), nx - 1);
          int32_t yy = std::min(std::max(y + dy, 0), ny - 1);
          s += g0[yy * nx + xx];
        }
      g[y * nx + x] = s / 9.0;
    }
  for (int32_t c = 0; c < n; ++c) K[c] = std::exp(2.0 * g[c]);
  auto harm = [](double a, double b) { return 2.0 * a * b / (a + b); };
  std::vector<int32_t> row(static_cast<size_t>(n) + 1, 0), col;
  std::vector<double> val;
  col.reserve(static_cast<size_t>(n) * 5);
  val.reserve(static_cast<size_t>(n) * 5);
  for (int32_t y = 0; y < ny; ++y)
    for (int32_t x = 0; x < nx; ++x) {
      const int32_t c = y * nx + x;
      const double kc = K[c];
      double fs = (y > 0) ? aniso * harm(kc, K[c - nx]) : aniso * 2.0 * kc;
      double fw = (x > 0) ? harm(kc, K[c - 1]) : 2.0 * kc;
      double fe = (x < nx - 1) ? harm(kc, K[c + 1]) : 2.0 * kc;
      double fn = (y < ny - 1) ? aniso * harm(kc, K[c + nx]) : aniso * 2.0 * kc;
      if (y > 0) { col.push_back(c - nx); val.push_back(-fs); }
      if (x > 0) { col.push_back(c - 1); val.push_back(-fw); }
      col.push_back(c);
      val.push_back(((fs + fw) + fe) + fn);
      if (x < nx - 1) { col.push_back(c + 1); val.push_back(-fe); }
      if (y < ny - 1) { col.push_back(c + nx); val.push_back(-fn); }
      row[c + 1] = static_cast<int32_t>(col.size());
    }
  WL_TRY(alloc_csr(n, static_cast<int64_t>(col.size()), out));
  std::memcpy(out->row, row.data(), sizeof(int32_t) * (n + 1));
  std::memcpy(out->col, col.data(), sizeof(int32_t) * col.size());
  std::memcpy(out->val, val.data(), sizeof(double) * val.size());
  return WL_OK;
}

int wl_rgg(int32_t n, uint64_t seed, double mean_degree, double wlo, double whi,
           double shift, wl_csr *out) {
  if (!out) return set_error(WL_ERR_PARAM, "null output");
  std::memset(out, 0, sizeof(*out));
  if (n <= 1 || !(mean_degree > 0)) return set_error(WL_ERR_PARAM, "bad RGG sizes");
  // Radius so that the expected number of neighbours in the (unbounded)
  // unit-density ball is mean_degree: n * 4/3 pi r^3 = mean_degree.
  const double r = std::cbrt(mean_degree / (static_cast<double>(n) * 4.0 / 3.0 *
                                            3.14159265358979323846));
  const double r2 = r * r;
  SplitMix64 rng(seed);
  std::vector<double> px(n), py(n), pz(n);
  for (int32_t i = 0; i < n; ++i) {
    px[i] = rng.uniform();
    py[i] = rng.uniform();
    pz[i] = rng.uniform();
  }
  int g = std::max(1, static_cast<int>(std::floor(1.0 / r)));
  auto cell = [&](double v) { return std::min(g - 1, static_cast<int>(v * g)); };
  const int64_t ncell = static_cast<int64_t>(g) * g * g;
  std::vector<int32_t> cstart(ncell + 1, 0), cidx(n);
  std::vector<int64_t> cid(n);
  for (int32_t i = 0; i < n; ++i) {
    cid[i] = (static_cast<int64_t>(cell(pz[i])) * g + cell(py[i])) * g + cell(px[i]);
    cstart[cid[i] + 1]++;
  }
  for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
  {
    std::vector<int32_t> fill(cstart.begin(), cstart.end() - 1);
    for (int32_t i = 0; i < n; ++i) cidx[fill[cid[i]]++] = i;
  }
  // Edge weight depends only on the unordered pair, so W is symmetric.
  auto weight = [&](int32_t a, int32_t b) {
    uint64_t lo = static_cast<uint64_t>(std::min(a, b));
    uint64_t hi = static_cast<uint64_t>(std::max(a, b));
    SplitMix64 h(seed ^ (hi * 0x100000001B3ULL + lo * 0xC2B2AE3D27D4EB4FULL));
    h.next();
    return wlo + (whi - wlo) * h.uniform();
  };
  std::vector<std::vector<std::pair<int32_t, double>>> adj(n);
  for (int32_t i = 0; i < n; ++i) {
    int cx = cell(px[i]), cy = cell(py[i]), cz = cell(pz[i]);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int xx = cx + dx, yy = cy + dy, zz = cz + dz;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= g || yy >= g || zz >= g) continue;
          int64_t c = (static_cast<int64_t>(zz) * g + yy) * g + xx;
          for (int32_t t = cstart[c]; t < cstart[c + 1]; ++t) {
            int32_t j = cidx[t];
            if (j == i) continue;
            double ddx = px[i] - px[j], ddy = py[i] - py[j], ddz = pz[i] - pz[j];
            if (ddx * ddx + ddy * ddy + ddz * ddz < r2) adj[i].push_back({j, weight(i, j)});
          }
        }
    std::sort(adj[i].begin(), adj[i].end());
  }
  int64_t nnz = n;
  for (int32_t i = 0; i < n; ++i) nnz += static_cast<int64_t>(adj[i].size());
  WL_TRY(alloc_csr(n, nnz, out));
  int64_t w = 0;
  out->row[0] = 0;
  for (int32_t i = 0; i < n; ++i) {
    double deg = 0.0;
    for (auto &e : adj[i]) deg += e.second;
    bool placed = false;
    for (auto &e : adj[i]) {
      if (!placed && e.first > i) {
        out->col[w] = i;
        out->val[w] = deg + shift;
        ++w;
        placed = true;
      }
      out->col[w] = e.first;
      out->val[w] = -e.second;
      ++w;
    }
    if (!placed) {
      out->col[w] = i;
      out->val[w] = deg + shift;
      ++w;
    }
    out->row[i + 1] = static_cast<int32_t>(w);
  }
  return WL_OK;
}

int wl_vector(int kind, uint64_t seed, int32_t n, double *out) {
  if (!out || n < 0) return set_error(WL_ERR_PARAM, "bad vector arguments");
  if (kind == 0) {
    for (int32_t i = 0; i < n; ++i) out[i] = 1.0;
  } else if (kind == 1) {
    Normal nrm(seed);
    for (int32_t i = 0; i < n; ++i) out[i] = nrm.next();
  } else if (kind == 2) {
    SplitMix64 rng(seed);
    for (int32_t i = 0; i < n; ++i) out[i] = 2.0 * rng.uniform() - 1.0;
  } else {
    return set_error(WL_ERR_PARAM, "unknown vector kind %d", kind);
  }
  return WL_OK;
}

}  // extern "C"
