// ref_mesh_shim.cpp -- C entry points around the reference's own Mesh class.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file against the
// reference tree (-I <reference>/include) into _ref/libmesh_ref.so; nothing
// of the reference is copied here.  It lets the tests compare
//   - the random grid of Mesh<Float>(solve_dim, dims) (include/util/mesh.hpp:85-124),
//     run with a chosen number of OpenMP threads, and
//   - the arrays Mesh<Float>(file) reads from a fixture file (mesh.hpp:51-80)
// with the oracle restatement and with the library.
#include <util/mesh.hpp>

#include <algorithm>
#include <vector>

namespace {

template <typename F>
void copy_out(const Mesh<F> &m, F *ds, F *dl, F *d, F *du, F *dw, F *x, F *u) {
  std::copy(m.ds().begin(), m.ds().end(), ds);
  std::copy(m.dl().begin(), m.dl().end(), dl);
  std::copy(m.d().begin(), m.d().end(), d);
  std::copy(m.du().begin(), m.du().end(), du);
  std::copy(m.dw().begin(), m.dw().end(), dw);
  std::copy(m.x().begin(), m.x().end(), x);
  if (u) std::copy(m.u().begin(), m.u().end(), u);
}

template <typename F>
int random_mesh(const int *dims, int ndims, int solvedim, int nthreads, F *ds, F *dl, F *d,
                F *du, F *dw, F *x) {
  omp_set_dynamic(0);
  omp_set_num_threads(nthreads);
  Mesh<F> m(static_cast<size_t>(solvedim), std::vector<int>(dims, dims + ndims));
  copy_out<F>(m, ds, dl, d, du, dw, x, nullptr);
  return 0;
}

template <typename F>
int load_mesh(const char *path, F *ds, F *dl, F *d, F *du, F *dw, F *x, F *u) {
  Mesh<F> m{std::filesystem::path(path)};
  copy_out<F>(m, ds, dl, d, du, dw, x, u);
  return static_cast<int>(m.solve_dim());
}

}  // namespace

extern "C" int ref_mesh_random_d(const int *dims, int ndims, int solvedim, int nthreads,
                                 double *ds, double *dl, double *d, double *du, double *dw,
                                 double *x) {
  return random_mesh<double>(dims, ndims, solvedim, nthreads, ds, dl, d, du, dw, x);
}

extern "C" int ref_mesh_random_s(const int *dims, int ndims, int solvedim, int nthreads,
                                 float *ds, float *dl, float *d, float *du, float *dw,
                                 float *x) {
  return random_mesh<float>(dims, ndims, solvedim, nthreads, ds, dl, d, du, dw, x);
}

extern "C" int ref_mesh_load_d(const char *path, double *ds, double *dl, double *d,
                               double *du, double *dw, double *x, double *u) {
  return load_mesh<double>(path, ds, dl, d, du, dw, x, u);
}

extern "C" int ref_mesh_load_s(const char *path, float *ds, float *dl, float *d, float *du,
                               float *dw, float *x, float *u) {
  return load_mesh<float>(path, ds, dl, d, du, dw, x, u);
}
