// bcmg_cli MATRIX SETTINGS [OUT]: the reference's solve_example
// (src/solve_example.cu:8-38) on this library's C ABI.  Reads a Matrix
// Market file and a 14-line settings file, solves A x = 1 from x0 = 0 and
// writes x one value per line with "%.14e" (Vector::printOnFile,
// src/matrix/vector.cu:444-466) to OUT (default x.txt).  Prints the #META
// lines of src/SOLVER/solver.cu:248-254 (format of src/utility/eval.cu:17-26).
// Options: --mixed selects the mixed-precision hierarchy.
#include <cstdio>
#include <cstring>
#include <vector>

#include "bcmg.h"

static void meta_int(const char *name, int v) { printf("#META %s int %d\n", name, v); }
static void meta_float(const char *name, double v) { printf("#META %s float %le\n", name, v); }

int main(int argc, char **argv) {
  const char *mpath = nullptr, *ppath = nullptr, *out = "x.txt";
  bool mixed = false;
  int pos = 0;
  for (int i = 1; i < argc; ++i) {
    if (std::strcmp(argv[i], "--mixed") == 0) {
      mixed = true;
      continue;
    }
    if (pos == 0) mpath = argv[i];
    if (pos == 1) ppath = argv[i];
    if (pos == 2) out = argv[i];
    ++pos;
  }
  if (!mpath || !ppath) {
    printf("matrix_path setting_file\n");
    return 1;
  }
  printf("READING INPUT MATRIX....:\n\n");
  bcmg_csr A;
  if (bcmg_read_matrix(mpath, 0, &A) != BCMG_OK) {
    fprintf(stderr, "error: %s\n", bcmg_last_error());
    return 1;
  }
  bcmg_params p;
  if (bcmg_params_from_file(ppath, &p) != BCMG_OK) {
    fprintf(stderr, "error: %s\n", bcmg_last_error());
    bcmg_csr_free(&A);
    return 1;
  }
  bcmg_ext e;
  bcmg_ext_default(&e);
  if (mixed) {
    e.precision = BCMG_PREC_MIXED;
    e.replace_every = 10;
  }
  printf("SOLVING....:\n\n");
  std::vector<double> b(A.n, 1.0), x(A.n, 0.0);
  bcmg_solve_info info;
  bcmg_status st = bcmg_solve_legacy(&A, &p, &e, b.data(), x.data(), &info);
  if (st != BCMG_OK) {
    fprintf(stderr, "error: %s: %s\n", bcmg_status_string(st), bcmg_last_error());
    bcmg_csr_free(&A);
    return 1;
  }
  meta_int("agg;hierarchy_levels_num", info.num_hrc);
  meta_float("agg;final_estimated_ratio", info.estimated_ratio);
  meta_int("sol;num_iteration", info.iters);
  meta_float("sol;residual", info.residual);
  meta_float("time;bootstrap_time", info.setup_ms);
  meta_float("time;solve_time", info.solve_ms);
  printf("bootstrap_time: %g sec \n", info.setup_ms / 1000);
  printf("solve_time: %g sec \n", info.solve_ms / 1000);
  FILE *f = fopen(out, "w");
  if (!f) {
    fprintf(stderr, "error: cannot write %s\n", out);
    bcmg_csr_free(&A);
    return 1;
  }
  for (double v : x) fprintf(f, "%.14e\n", v);
  fclose(f);
  bcmg_csr_free(&A);
  return 0;
}
