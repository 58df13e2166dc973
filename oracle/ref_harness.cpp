// CPU oracle harness over the REFERENCE VBCSR implementation.
//
// Test infrastructure only: this file is compiled against the reference's own
// headers (vbcsr/core/*.hpp, header-only C++17 + OpenMP) into
// oracle/_ref/libvbcsr_ref.so by oracle/build_ref.sh.  It exposes a flat C ABI
// so that tests/ and bench.py's reference arm can drive the reference's
// BlockSpMat with exactly the inputs the GPU library receives.  Nothing in the
// shipped library links or loads it.
//
// Reference entry points exercised (paths relative to the reference repo):
//   construction   vbcsr/core/dist_graph.hpp:167 construct_serial,
//                  vbcsr/core/block_csr.hpp:613 add_block, :861 assemble
//   mult / adjoint vbcsr/core/block_csr.hpp:985-1050
//   spmm           vbcsr/core/block_csr.hpp:1530 -> detail/ops/spmm/vbcsr.hpp:70
//   rarh_upper, rhar_upper, square_polynomial_upper
//                  vbcsr/core/block_csr.hpp:1803-1853 -> detail/ops/spmm/
//                  rarh.hpp, rhar.hpp, square_polynomial.hpp
//   filter_blocks  vbcsr/core/block_csr.hpp:1399
//   axpby/scale/shift  vbcsr/core/block_csr.hpp:1053,1250,1289
//   transpose      vbcsr/core/block_csr.hpp:2047
//   set_random     vbcsr/core/dist_multivector.hpp:335
//   KPM recurrence examples/ex08_graphene_dos.py:66-156 (driven here through
//                  the same DistMultiVector ops the Python loop calls)
//   propagation    examples/ex09_graphene_dynamics.py:102-133
#include <block_csr.hpp>

#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <omp.h>
#include <vector>

using namespace vbcsr;
using cplx = std::complex<double>;

namespace {

struct RefMat {
  int is_complex = 0;
  DistGraph* graph = nullptr;  // graph we created (matrix may later own another)
  std::unique_ptr<BlockSpMat<double>> d;
  std::unique_ptr<BlockSpMat<cplx>> z;
  ~RefMat() {
    d.reset();
    z.reset();
    delete graph;
  }
};

template <typename T>
BlockSpMat<T>& mat_of(RefMat* m);
template <>
BlockSpMat<double>& mat_of<double>(RefMat* m) { return *m->d; }
template <>
BlockSpMat<cplx>& mat_of<cplx>(RefMat* m) { return *m->z; }

template <typename T>
void fill_blocks(BlockSpMat<T>& M, int n, const int* bs, const int* rp, const int* ci,
                 const T* vals) {
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    for (int s = rp[i]; s < rp[i + 1]; ++s) {
      const int j = ci[s];
      M.add_block(i, j, vals + off, bs[i], bs[j], AssemblyMode::INSERT);
      off += static_cast<size_t>(bs[i]) * bs[j];
    }
  }
  M.assemble();
}

template <typename T>
RefMat* wrap(BlockSpMat<T>&& M, int is_complex);
template <>
RefMat* wrap<double>(BlockSpMat<double>&& M, int) {
  auto* r = new RefMat();
  r->is_complex = 0;
  r->d.reset(new BlockSpMat<double>(std::move(M)));
  return r;
}
template <>
RefMat* wrap<cplx>(BlockSpMat<cplx>&& M, int) {
  auto* r = new RefMat();
  r->is_complex = 1;
  r->z.reset(new BlockSpMat<cplx>(std::move(M)));
  return r;
}

template <typename T>
void do_mult(RefMat* m, const T* x, T* y, bool adjoint) {
  auto& M = mat_of<T>(m);
  DistVector<T> vx(M.graph), vy(M.graph);
  std::memcpy(vx.local_data(), x, sizeof(T) * vx.size());
  if (adjoint) M.mult_adjoint(vx, vy); else M.mult(vx, vy);
  std::memcpy(y, vy.local_data(), sizeof(T) * vy.size());
}

template <typename T>
void load_mv(DistMultiVector<T>& V, const T* X, int k) {
  for (int r = 0; r < V.local_rows; ++r)
    for (int c = 0; c < k; ++c) V(r, c) = X[static_cast<size_t>(r) * k + c];
}
template <typename T>
void store_mv(DistMultiVector<T>& V, T* X, int k) {
  for (int r = 0; r < V.local_rows; ++r)
    for (int c = 0; c < k; ++c) X[static_cast<size_t>(r) * k + c] = V(r, c);
}

template <typename T>
void do_mult_dense(RefMat* m, int k, const T* X, T* Y, bool adjoint) {
  auto& M = mat_of<T>(m);
  DistMultiVector<T> vx(M.graph, k), vy(M.graph, k);
  load_mv(vx, X, k);
  if (adjoint) M.mult_dense_adjoint(vx, vy); else M.mult_dense(vx, vy);
  store_mv(vy, Y, k);
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int ref_get_threads(void) { return omp_get_max_threads(); }

// values: slot-ordered row-major blocks; complex as interleaved (re, im).
void* ref_mat_create(int n_blocks, const int* block_sizes, const int* row_ptr,
                     const int* col_ind, const void* values, int is_complex) {
  std::vector<int> bs(block_sizes, block_sizes + n_blocks);
  std::vector<std::vector<int>> adj(n_blocks);
  for (int i = 0; i < n_blocks; ++i) adj[i].assign(col_ind + row_ptr[i], col_ind + row_ptr[i + 1]);
  auto* r = new RefMat();
  r->is_complex = is_complex;
  r->graph = new DistGraph(MPI_COMM_NULL);
  r->graph->construct_serial(n_blocks, bs, adj);
  if (is_complex) {
    r->z.reset(new BlockSpMat<cplx>(r->graph));
    fill_blocks(*r->z, n_blocks, block_sizes, row_ptr, col_ind, static_cast<const cplx*>(values));
  } else {
    r->d.reset(new BlockSpMat<double>(r->graph));
    fill_blocks(*r->d, n_blocks, block_sizes, row_ptr, col_ind, static_cast<const double*>(values));
  }
  return r;
}

void ref_mat_free(void* h) { delete static_cast<RefMat*>(h); }

static const DistGraph* graph_of(RefMat* m) { return m->is_complex ? m->z->graph : m->d->graph; }

long long ref_mat_nnzb(void* h) { return static_cast<long long>(graph_of(static_cast<RefMat*>(h))->adj_ind.size()); }
int ref_mat_rows(void* h) { return static_cast<int>(graph_of(static_cast<RefMat*>(h))->adj_ptr.size()) - 1; }
long long ref_mat_nnz(void* h) {
  auto* m = static_cast<RefMat*>(h);
  return m->is_complex ? static_cast<long long>(m->z->local_scalar_nnz()) : static_cast<long long>(m->d->local_scalar_nnz());
}
int ref_mat_kind(void* h) {
  auto* m = static_cast<RefMat*>(h);
  return static_cast<int>(m->is_complex ? m->z->matrix_kind() : m->d->matrix_kind());
}

// row_ptr (n+1) and GLOBAL col_ind (nnzb).
void ref_mat_structure(void* h, int* row_ptr, int* col_ind) {
  const DistGraph* g = graph_of(static_cast<RefMat*>(h));
  const int n = static_cast<int>(g->adj_ptr.size()) - 1;
  for (int i = 0; i <= n; ++i) row_ptr[i] = g->adj_ptr[i];
  for (size_t s = 0; s < g->adj_ind.size(); ++s) col_ind[s] = g->get_global_index(g->adj_ind[s]);
}

void ref_mat_values(void* h, void* out) {
  auto* m = static_cast<RefMat*>(h);
  if (m->is_complex) {
    auto v = m->z->get_values();
    std::memcpy(out, v.data(), v.size() * sizeof(cplx));
  } else {
    auto v = m->d->get_values();
    std::memcpy(out, v.data(), v.size() * sizeof(double));
  }
}

void ref_mult(void* h, const void* x, void* y) {
  auto* m = static_cast<RefMat*>(h);
  if (m->is_complex) do_mult(m, static_cast<const cplx*>(x), static_cast<cplx*>(y), false);
  else do_mult(m, static_cast<const double*>(x), static_cast<double*>(y), false);
}
void ref_mult_adjoint(void* h, const void* x, void* y) {
  auto* m = static_cast<RefMat*>(h);
  if (m->is_complex) do_mult(m, static_cast<const cplx*>(x), static_cast<cplx*>(y), true);
  else do_mult(m, static_cast<const double*>(x), static_cast<double*>(y), true);
}
// X, Y: dense row-major N x k (no padding).
void ref_mult_dense(void* h, int k, const void* X, void* Y) {
  auto* m = static_cast<RefMat*>(h);
  if (m->is_complex) do_mult_dense(m, k, static_cast<const cplx*>(X), static_cast<cplx*>(Y), false);
  else do_mult_dense(m, k, static_cast<const double*>(X), static_cast<double*>(Y), false);
}
void ref_mult_dense_adjoint(void* h, int k, const void* X, void* Y) {
  auto* m = static_cast<RefMat*>(h);
  if (m->is_complex) do_mult_dense(m, k, static_cast<const cplx*>(X), static_cast<cplx*>(Y), true);
  else do_mult_dense(m, k, static_cast<const double*>(X), static_cast<double*>(Y), true);
}

// Repeated SpMV, for the timed CPU baseline.
void ref_mult_repeat(void* h, const double* x, double* y, int repeats) {
  auto* m = static_cast<RefMat*>(h);
  auto& M = *m->d;
  DistVector<double> vx(M.graph), vy(M.graph);
  std::memcpy(vx.local_data(), x, sizeof(double) * vx.size());
  for (int r = 0; r < repeats; ++r) M.mult(vx, vy);
  std::memcpy(y, vy.local_data(), sizeof(double) * vy.size());
}

void* ref_spmm(void* a, void* b, double threshold, int transA, int transB) {
  auto* A = static_cast<RefMat*>(a);
  auto* B = static_cast<RefMat*>(b);
  if (A->is_complex) return wrap<cplx>(A->z->spmm(*B->z, threshold, transA != 0, transB != 0), 1);
  return wrap<double>(A->d->spmm(*B->d, threshold, transA != 0, transB != 0), 0);
}

void* ref_spmm_hermitian(void* a, void* b, double threshold, int transA) {
  auto* A = static_cast<RefMat*>(a);
  auto* B = static_cast<RefMat*>(b);
  if (A->is_complex) return wrap<cplx>(A->z->spmm_hermitian(*B->z, threshold, transA != 0), 1);
  return wrap<double>(A->d->spmm_hermitian(*B->d, threshold, transA != 0), 0);
}

// The fused triple products (block_csr.hpp:1803-1853): upper block triangle.
void* ref_rarh_upper(void* a, void* b, double threshold) {
  auto* A = static_cast<RefMat*>(a);
  auto* B = static_cast<RefMat*>(b);
  if (A->is_complex) return wrap<cplx>(A->z->rarh_upper(*B->z, threshold), 1);
  return wrap<double>(A->d->rarh_upper(*B->d, threshold), 0);
}

void* ref_rhar_upper(void* a, void* b, double threshold) {
  auto* A = static_cast<RefMat*>(a);
  auto* B = static_cast<RefMat*>(b);
  if (A->is_complex) return wrap<cplx>(A->z->rhar_upper(*B->z, threshold), 1);
  return wrap<double>(A->d->rhar_upper(*B->d, threshold), 0);
}

void* ref_square_polynomial_upper(void* a, double c2r, double c2i, double c1r, double c1i, double c0r, double c0i,
                                  double threshold) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex)
    return wrap<cplx>(A->z->square_polynomial_upper(cplx(c2r, c2i), cplx(c1r, c1i), cplx(c0r, c0i), threshold), 1);
  return wrap<double>(A->d->square_polynomial_upper(c2r, c1r, c0r, threshold), 0);
}

void* ref_transpose(void* a) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) return wrap<cplx>(A->z->transpose(), 1);
  return wrap<double>(A->d->transpose(), 0);
}

void* ref_duplicate(void* a) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) return wrap<cplx>(A->z->duplicate(true), 1);
  return wrap<double>(A->d->duplicate(true), 0);
}

void ref_filter_blocks(void* a, double threshold) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) A->z->filter_blocks(threshold); else A->d->filter_blocks(threshold);
}

void ref_scale(void* a, double re, double im) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) A->z->scale(cplx(re, im)); else A->d->scale(re);
}
void ref_shift(void* a, double re, double im) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) A->z->shift(cplx(re, im)); else A->d->shift(re);
}
// Y <- alpha * X + beta * Y
void ref_axpby(void* y, double are, double aim, void* x, double bre, double bim) {
  auto* Y = static_cast<RefMat*>(y);
  auto* X = static_cast<RefMat*>(x);
  if (Y->is_complex) Y->z->axpby(cplx(are, aim), *X->z, cplx(bre, bim));
  else Y->d->axpby(are, *X->d, bre);
}

double ref_block_density(void* a) {
  auto* A = static_cast<RefMat*>(a);
  return A->is_complex ? A->z->get_block_density() : A->d->get_block_density();
}

// Block Frobenius norms in slot order.
void ref_block_norms(void* a, double* out) {
  auto* A = static_cast<RefMat*>(a);
  const auto& v = A->is_complex ? A->z->get_block_norms() : A->d->get_block_norms();
  std::memcpy(out, v.data(), v.size() * sizeof(double));
}

// DistMultiVector::set_random with the scalar type's default kind; out is
// dense row-major N x k.
void ref_set_random(void* a, int k, unsigned long long seed, int normalize, void* out) {
  auto* A = static_cast<RefMat*>(a);
  if (A->is_complex) {
    DistMultiVector<cplx> V(A->z->graph, k);
    V.set_random(seed, normalize != 0);
    store_mv(V, static_cast<cplx*>(out), k);
  } else {
    DistMultiVector<double> V(A->d->graph, k);
    V.set_random(seed, normalize != 0);
    store_mv(V, static_cast<double*>(out), k);
  }
}

// Unnormalised KPM moments mu_n = sum_r Re <v0_r | T_n(H) | v0_r>, n < M, with
// the three-term recurrence of examples/ex08_graphene_dos.py:89-114 run on the
// reference's DistMultiVector ops (mult_dense, scale, axpy, bdot).  H is used
// as given (the caller scales it).  V0: dense row-major N x R.
void ref_kpm_moments(void* h, int R, int M, const double* V0, double* moments) {
  auto* m = static_cast<RefMat*>(h);
  auto& H = *m->d;
  DistMultiVector<double> v0(H.graph, R), vprev(H.graph, R), vcur(H.graph, R), vnext(H.graph, R);
  load_mv(v0, V0, R);
  auto sum_re = [](const std::vector<double>& d) { double s = 0; for (double x : d) s += x; return s; };
  if (M > 0) moments[0] = sum_re(v0.bdot(v0));
  if (M < 2) return;
  H.mult_dense(v0, vcur);
  moments[1] = sum_re(v0.bdot(vcur));
  vprev.copy_from(v0);
  for (int n = 2; n < M; ++n) {
    H.mult_dense(vcur, vnext);
    vnext.scale(2.0);
    vnext.axpy(-1.0, vprev);
    moments[n] = sum_re(v0.bdot(vnext));
    vprev.swap(vcur);
    vcur.swap(vnext);
  }
}

// psi_out = sum_n c_n T_n(H) psi for complex H, the loop of
// examples/ex09_graphene_dynamics.py:102-133 (H already scaled).  coeffs are
// interleaved complex.
void ref_cheb_apply(void* h, int M, const double* coeffs_ri, const void* psi, void* out) {
  auto* m = static_cast<RefMat*>(h);
  auto& H = *m->z;
  const cplx* c = reinterpret_cast<const cplx*>(coeffs_ri);
  DistVector<cplx> v0(H.graph), v1(H.graph), v2(H.graph), res(H.graph);
  const int n = v0.size();
  std::memcpy(v0.local_data(), psi, sizeof(cplx) * n);
  for (int i = 0; i < n; ++i) res[i] = v0[i] * c[0];
  if (M > 1) {
    H.mult(v0, v1);
    for (int i = 0; i < n; ++i) res[i] += v1[i] * c[1];
  }
  for (int k = 2; k < M; ++k) {
    H.mult(v1, v2);
    for (int i = 0; i < n; ++i) {
      v2[i] = 2.0 * v2[i] - v0[i];
      res[i] += v2[i] * c[k];
    }
    std::swap(v0.data, v1.data);
    std::swap(v1.data, v2.data);
  }
  std::memcpy(out, res.local_data(), sizeof(cplx) * n);
}

}  // extern "C"
