// vbcsr_core: the host core of the B200 engine, exported under the module
// name and class/method names of the reference's pybind extension
// (vbcsr/pybind_vbcsr.cpp:126-505) so that the reference's Python package,
// or this repository's mirror of it (vbcsr_b200), runs on top of it.
//
// The core keeps authoritative HOST mirrors of every matrix and vector (the
// reference hands numpy views of its buffers to Python, multivector.py:28-29,
// 89-111) next to DEVICE copies owned through the C ABI of
// include/vbcsr_b200.h.  Each object tracks which side is current; a Python
// buffer access brings the host copy up to date and marks the device copy
// stale, a device operation does the reverse.  All device work runs on one
// non-blocking stream; host copies synchronise it.
//
// Scope: the serial (single-rank, single-GPU) case of the reference --
// DistGraph::construct_serial / construct_distributed with all blocks owned
// (vbcsr/core/dist_graph.hpp:167-469).  Multi-rank communicators, MPI
// redistribution, submatrix extraction and the graph matrix functions (spmf)
// are not part of the engine and raise.
#include <cuda_runtime.h>
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "vbcsr_b200.h"

namespace py = pybind11;
using cplx = std::complex<double>;

namespace {

enum class AssemblyMode { INSERT = 0, ADD = 1 };
enum class RedistOp { Copy = 0, Sum = 1 };
enum class PhaseConvention { R_ONLY = 0, R_AND_POSITION = 1 };
// Import-time placeholders of the reference's atomic-structure classes.
struct AtomicDataStub {};
struct ImageContainerStub {};
struct ImageContainerComplexStub {};

cudaStream_t g_stream = nullptr;

cudaStream_t stream() {
  if (!g_stream) {
    if (cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking) != cudaSuccess)
      throw std::runtime_error("vbcsr_core: no CUDA device available (cudaStreamCreate failed)");
    // keep freed blocks cached in the default pool (stream-ordered reuse)
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  return g_stream;
}

void check(int rc, const char* what) {
  if (rc != 0) throw std::runtime_error(std::string(what) + ": " + vbg_last_error());
}
void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T> constexpr int dtype_code();
template <> constexpr int dtype_code<double>() { return VBG_F64; }
template <> constexpr int dtype_code<cplx>() { return VBG_C128; }

// Device allocation, stream ordered.
struct DBuf {
  void* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, stream());
    p = nullptr;
    n = 0;
  }
  void ensure(size_t bytes) {
    if (p && bytes <= n) return;
    release();
    cuda_check(cudaMallocAsync(&p, std::max<size_t>(bytes, 16), stream()), "cudaMallocAsync");
    n = bytes;
  }
};

// ------------------------------------------------------------------ graph
// Serial DistGraph: every block owned, local index == global index, each
// row's neighbours sorted (dist_graph.hpp:299).
struct Graph {
  int n = 0;
  std::vector<int> bsz, row_ptr{0}, col_ind;
  std::vector<int64_t> scal_off{0};
  // block structure only, per scalar type (device vector ops: the random
  // fill draws Rademacher signs for F64 and phases for C128)
  vbg_matrix* shape_handle[2] = {nullptr, nullptr};

  Graph() = default;
  Graph(const Graph& o) : n(o.n), bsz(o.bsz), row_ptr(o.row_ptr), col_ind(o.col_ind), scal_off(o.scal_off) {}
  ~Graph() { drop_shapes(); }
  void drop_shapes() {
    for (vbg_matrix*& h : shape_handle) {
      if (h) vbg_matrix_destroy(h);
      h = nullptr;
    }
  }

  void finish() {
    scal_off.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) scal_off[i + 1] = scal_off[i] + bsz[i];
    drop_shapes();
  }
  int64_t N() const { return scal_off[n]; }
  int64_t nnzb() const { return (int64_t)col_ind.size(); }

  void set_rows(int nb, const std::vector<int>& sizes, const int64_t* aptr, const int* aind) {
    if ((int)sizes.size() != nb) throw std::runtime_error("DistGraph: block size count does not match block count");
    for (int b : sizes)
      if (b < 1) throw std::runtime_error("DistGraph: block sizes must be >= 1");
    n = nb;
    bsz = sizes;
    row_ptr.assign(n + 1, 0);
    col_ind.clear();
    for (int i = 0; i < n; ++i) {
      if (aptr[i + 1] < aptr[i]) throw std::runtime_error("construct_distributed_flat: adj_ptr not monotone");
      std::vector<int> cols(aind + aptr[i], aind + aptr[i + 1]);
      for (int c : cols)
        if (c < 0 || c >= n) throw std::runtime_error("DistGraph: neighbour index out of range");
      std::sort(cols.begin(), cols.end());
      col_ind.insert(col_ind.end(), cols.begin(), cols.end());
      row_ptr[i + 1] = (int)col_ind.size();
    }
    finish();
  }

  void set_lists(int nb, const std::vector<int>& sizes, const std::vector<std::vector<int>>& adj) {
    if ((int)adj.size() != nb) throw std::runtime_error("DistGraph: adjacency size does not match block count");
    std::vector<int64_t> ptr(nb + 1, 0);
    std::vector<int> ind;
    for (int i = 0; i < nb; ++i) {
      ind.insert(ind.end(), adj[i].begin(), adj[i].end());
      ptr[i + 1] = (int64_t)ind.size();
    }
    set_rows(nb, sizes, ptr.data(), ind.data());
  }

  int slot(int row, int col) const {
    auto b = col_ind.begin() + row_ptr[row], e = col_ind.begin() + row_ptr[row + 1];
    auto it = std::lower_bound(b, e, col);
    if (it == e || *it != col) return -1;
    return (int)(it - col_ind.begin());
  }
  std::vector<int64_t> slot_offsets() const {
    std::vector<int64_t> off(col_ind.size() + 1, 0);
    for (int i = 0; i < n; ++i)
      for (int s = row_ptr[i]; s < row_ptr[i + 1]; ++s) off[s + 1] = off[s] + (int64_t)bsz[i] * bsz[col_ind[s]];
    return off;
  }
  int64_t nnz() const { return slot_offsets().back(); }
  bool same_owned_structure(const Graph& o) const { return n == o.n && bsz == o.bsz; }

  vbg_matrix* shape(int dtype) {
    vbg_matrix*& h = shape_handle[dtype == VBG_C128 ? 1 : 0];
    if (!h) {
      std::vector<int> rp(n + 1, 0);
      check(vbg_matrix_create(&h, dtype, n, bsz.data(), rp.data(), nullptr, nullptr, stream()), "vbg_matrix_create");
    }
    return h;
  }
};

using GraphPtr = std::shared_ptr<Graph>;

GraphPtr graph_from_device(const vbg_matrix* m) {
  int n = 0;
  int64_t nnzb = 0;
  check(vbg_matrix_info(m, nullptr, &n, &nnzb, nullptr, nullptr, nullptr), "vbg_matrix_info");
  auto g = std::make_shared<Graph>();
  g->n = n;
  g->row_ptr.assign(n + 1, 0);
  g->col_ind.assign(std::max<int64_t>(nnzb, 1), 0);
  g->bsz.assign(std::max(n, 1), 0);
  check(vbg_matrix_get_structure(m, g->row_ptr.data(), g->col_ind.data(), g->bsz.data()), "vbg_matrix_get_structure");
  g->col_ind.resize(nnzb);
  g->bsz.resize(n);
  g->finish();
  return g;
}

// ---------------------------------------------------------------- vectors
// One implementation for DistVector (k = 1, ld = 1) and DistMultiVector
// (row-major, ld = k rounded up to 64 bytes, zero pad lanes;
// dist_multivector.hpp:24-67).
template <typename T>
struct Vec {
  GraphPtr g;
  int k = 1, ld = 1;
  bool multi = false;
  int64_t rows = 0;
  std::vector<T> host;
  DBuf dev;
  bool host_ok = true, dev_ok = false;

  static int ld_for(int k) {
    const int per_line = 64 / (int)sizeof(T);
    return ((k + per_line - 1) / per_line) * per_line;
  }
  Vec(GraphPtr gr, int kk, bool mv) : g(std::move(gr)), k(kk), multi(mv) {
    if (k < 1) throw std::runtime_error("DistMultiVector: num_vectors must be >= 1");
    ld = mv ? ld_for(k) : 1;
    rows = g->N();
    host.assign((size_t)rows * ld, T(0));
  }
  size_t bytes() const { return (size_t)rows * ld * sizeof(T); }
  void to_host() {
    if (host_ok) return;
    cuda_check(cudaMemcpyAsync(host.data(), dev.p, bytes(), cudaMemcpyDeviceToHost, stream()), "D2H");
    cuda_check(cudaStreamSynchronize(stream()), "sync");
    host_ok = true;
  }
  void to_device() {
    if (dev_ok) return;
    dev.ensure(bytes());
    cuda_check(cudaMemcpyAsync(dev.p, host.data(), bytes(), cudaMemcpyHostToDevice, stream()), "H2D");
    dev_ok = true;
  }
  void* read() {
    to_device();
    return dev.p;
  }
  void* readwrite() {
    to_device();
    host_ok = false;
    return dev.p;
  }
  // Output of a device op that writes every element (pads included).
  void* write_all() {
    dev.ensure(bytes());
    dev_ok = true;
    host_ok = false;
    return dev.p;
  }
  // Python buffer access: the host copy becomes the authoritative one.
  T* host_for_python() {
    to_host();
    dev_ok = false;
    return host.data();
  }
  void copy_from(const Vec& o) {
    if (o.rows != rows || o.k != k)
      throw std::runtime_error(multi ? "DistMultiVector::copy_from: size mismatch" : "DistVector::copy_from: size mismatch");
    if (o.dev_ok) {
      dev.ensure(bytes());
      cuda_check(cudaMemcpyAsync(dev.p, o.dev.p, bytes(), cudaMemcpyDeviceToDevice, stream()), "D2D");
      dev_ok = true;
      host_ok = false;
    } else {
      host = o.host;
      host_ok = true;
      dev_ok = false;
    }
  }
  void set_constant(T val) {
    to_host();
    for (int64_t r = 0; r < rows; ++r)
      for (int c = 0; c < k; ++c) host[(size_t)r * ld + c] = val;
    dev_ok = false;
  }
  void scale(T a) {
    const cplx z(a);
    check(vbg_mv_scale(dtype_code<T>(), rows, k, ld, z.real(), z.imag(), readwrite(), stream()), "scale");
  }
  void axpby(T a, const Vec& x, T b) {
    if (x.rows != rows || x.k != k) throw std::runtime_error("axpby: dimension mismatch");
    const void* xp = const_cast<Vec&>(x).read();
    const cplx za(a), zb(b);
    check(vbg_mv_axpby(dtype_code<T>(), rows, k, ld, za.real(), za.imag(), xp, zb.real(), zb.imag(), readwrite(),
                       stream()),
          "axpby");
  }
  void pointwise(const Vec& y, bool y_is_vector) {
    const void* yp = const_cast<Vec&>(y).read();
    check(vbg_mv_pointwise(dtype_code<T>(), rows, k, ld, yp, y_is_vector ? 1 : 0, readwrite(), stream()),
          "pointwise_mult");
  }
  std::vector<T> bdot(const Vec& x) const {
    if (x.k != k || x.rows != rows) throw std::runtime_error("Dimension mismatch in bdot");
    DBuf out;
    out.ensure(k * sizeof(T));
    const void* a = const_cast<Vec&>(*this).read();
    const void* b = const_cast<Vec&>(x).read();
    check(vbg_mv_bdot(dtype_code<T>(), rows, k, ld, a, b, out.p, stream()), "bdot");
    std::vector<T> res(k);
    cuda_check(cudaMemcpyAsync(res.data(), out.p, k * sizeof(T), cudaMemcpyDeviceToHost, stream()), "D2H");
    cuda_check(cudaStreamSynchronize(stream()), "sync");
    return res;
  }
  void set_random(uint64_t seed, bool normalize) {
    check(vbg_mv_set_random(g->shape(dtype_code<T>()), k, ld, seed, normalize ? 1 : 0, write_all(), stream()), "set_random");
  }
};

// Distinct C++ types for the two Python classes of each scalar type.
template <typename T, bool MULTI>
struct DV : Vec<T> {
  DV(GraphPtr g, int k) : Vec<T>(std::move(g), k, MULTI) {}
};

// A DistVector or DistMultiVector of scalar type T passed as a Python object.
template <typename T>
Vec<T>& vec_of(py::object o) {
  if (py::isinstance<DV<T, true>>(o)) return o.cast<DV<T, true>&>();
  if (py::isinstance<DV<T, false>>(o)) return o.cast<DV<T, false>&>();
  throw std::runtime_error("expected a DistVector or DistMultiVector of the matrix's scalar type");
}

template <typename T>
py::array_t<T> to_array(const std::vector<T>& v) {
  py::array_t<T> a((py::ssize_t)v.size());
  if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), sizeof(T) * v.size());
  return a;
}

// ---------------------------------------------------------------- matrix
template <typename T>
struct Mat {
  GraphPtr g;
  std::vector<T> host;
  bool host_ok = true, dev_ok = false;
  vbg_matrix* dm = nullptr;

  explicit Mat(GraphPtr gr) : g(std::move(gr)) { host.assign(g->nnz(), T(0)); }
  Mat(GraphPtr gr, int) : g(std::move(gr)) {}
  Mat(const Mat&) = delete;
  ~Mat() {
    if (dm) vbg_matrix_destroy(dm);
  }

  void ensure_device() {
    if (!dm) {
      check(vbg_matrix_create(&dm, dtype_code<T>(), g->n, g->bsz.data(), g->row_ptr.data(), g->col_ind.data(),
                              host.data(), stream()),
            "vbg_matrix_create");
      dev_ok = true;
      return;
    }
    if (!dev_ok) {
      check(vbg_matrix_set_values(dm, host.data(), stream()), "vbg_matrix_set_values");
      dev_ok = true;
    }
  }
  void ensure_host() {
    if (host_ok) return;
    host.resize(g->nnz());
    check(vbg_matrix_get_values(dm, host.data(), stream()), "vbg_matrix_get_values");
    host_ok = true;
  }
  void device_modified() { host_ok = false; }
  void host_modified() { dev_ok = false; }
  // After an operation that may have changed the device pattern.
  void adopt_device_structure() {
    int n = 0;
    int64_t nnzb = 0;
    check(vbg_matrix_info(dm, nullptr, &n, &nnzb, nullptr, nullptr, nullptr), "vbg_matrix_info");
    bool same = nnzb == g->nnzb();
    if (same) {
      std::vector<int> rp(n + 1), ci(std::max<int64_t>(nnzb, 1));
      check(vbg_matrix_get_structure(dm, rp.data(), ci.data(), nullptr), "vbg_matrix_get_structure");
      ci.resize(nnzb);
      same = rp == g->row_ptr && ci == g->col_ind;
    }
    if (!same) g = graph_from_device(dm);
    host_ok = false;
    dev_ok = true;
  }
  static std::unique_ptr<Mat> wrap_device(vbg_matrix* d) {
    auto m = std::unique_ptr<Mat>(new Mat(graph_from_device(d), 0));
    m->dm = d;
    m->host_ok = false;
    m->dev_ok = true;
    return m;
  }
  void check_vec(const Vec<T>& x) const {
    if (!g->same_owned_structure(*x.g))
      throw std::runtime_error(
          "DistVector::bind_to_graph: graph mismatch - target graph has a different owned block structure "
          "(partition or block sizes)");
  }
  void mult(Vec<T>& x, Vec<T>& y, bool adjoint) {
    check_vec(x);
    check_vec(y);
    ensure_device();
    const void* xp = x.read();
    if (!x.multi) {
      void* yp = y.write_all();
      check(adjoint ? vbg_spmv_adjoint(dm, xp, yp, stream()) : vbg_spmv(dm, xp, yp, stream()), "mult");
    } else {
      if (x.k != y.k) throw std::runtime_error("mult_dense: num_vectors mismatch");
      void* yp = y.write_all();
      check(adjoint ? vbg_spmm_adjoint(dm, x.k, x.ld, xp, yp, stream()) : vbg_spmm(dm, x.k, x.ld, xp, yp, stream()),
            "mult_dense");
    }
  }
  void add_block(int r, int c, py::array_t<T, py::array::c_style | py::array::forcecast> data, AssemblyMode mode) {
    if (data.ndim() != 2) throw std::runtime_error("add_block: array must be 2D");
    const int s = (r >= 0 && r < g->n && c >= 0 && c < g->n) ? g->slot(r, c) : -1;
    if (s < 0) {
      std::cerr << "Warning: Block (row=" << r << ", col=" << c << ") not found in local graph. Ignoring." << std::endl;
      return;
    }
    const int rd = g->bsz[r], cd = g->bsz[c];
    if (data.shape(0) != rd || data.shape(1) != cd)
      throw std::runtime_error("add_block: block dimensions do not match the graph");
    ensure_host();
    const int64_t off = g->slot_offsets()[s];
    const T* src = data.data();
    for (int e = 0; e < rd * cd; ++e) {
      if (mode == AssemblyMode::INSERT) host[off + e] = src[e];
      else host[off + e] += src[e];
    }
    host_modified();
  }
  // Bulk fill of every block in slot order: this engine's fast path for the
  // per-block add_block loops of create_random / from_scipy.
  void set_values(py::array_t<T, py::array::c_style | py::array::forcecast> v) {
    if ((int64_t)v.size() != g->nnz()) throw std::runtime_error("set_values: size mismatch");
    ensure_host();
    std::memcpy(host.data(), v.data(), sizeof(T) * v.size());
    host_modified();
  }
};

using MatD = Mat<double>;

template <typename T, bool MULTI>
void bind_vector(py::module& m, const char* name) {
  using V = DV<T, MULTI>;
  py::class_<V> cls(m, name, py::buffer_protocol());
  if (MULTI)
    cls.def(py::init([](GraphPtr g, int k) { return std::make_unique<V>(g, k); }), py::keep_alive<1, 2>());
  else
    cls.def(py::init([](GraphPtr g) { return std::make_unique<V>(g, 1); }), py::keep_alive<1, 2>());
  cls.def("sync_ghosts", [](V&) {})
      .def("reduce_ghosts", [](V&) {})
      .def("set_constant", [](V& v, T val) { v.set_constant(val); })
      .def("scale", [](V& v, T a) { v.scale(a); })
      .def("axpy", [](V& y, T a, const V& x) { y.axpby(a, x, T(1)); })
      .def("axpby", [](V& y, T a, const V& x, T b) { y.axpby(a, x, b); })
      .def("duplicate", [](const V& v) {
        auto d = std::make_unique<V>(v.g, v.k);
        d->copy_from(v);
        return d;
      })
      .def("copy_from", [](V& a, const V& b) { a.copy_from(b); })
      .def("set_random", [](V& v, uint64_t seed, bool normalize) { v.set_random(seed, normalize); },
           py::arg("seed"), py::arg("normalize") = true)
      .def("reset_comm_stats", [](V&) {})
      .def_property_readonly("comm_seconds", [](const V&) { return 0.0; })
      .def_property_readonly("comm_calls", [](const V&) { return 0; })
      .def_buffer([](V& v) -> py::buffer_info {
        T* p = v.host_for_python();
        if (!MULTI)
          return py::buffer_info(p, sizeof(T), py::format_descriptor<T>::format(), 1, {(size_t)v.rows}, {sizeof(T)});
        return py::buffer_info(p, sizeof(T), py::format_descriptor<T>::format(), 2, {(size_t)v.rows, (size_t)v.k},
                               {sizeof(T) * (size_t)v.ld, sizeof(T)});
      });
  if (MULTI) {
    cls.def("pointwise_mult", [](V& a, const V& b) {
         if (b.k != a.k) throw std::runtime_error("pointwise_mult: shape mismatch");
         a.pointwise(b, false);
       })
        .def("pointwise_mult_vec", [](V& a, const DV<T, false>& b) { a.pointwise(b, true); })
        .def("bdot", [](const V& a, const V& b) { return a.bdot(b); })
        .def_property_readonly("local_rows", [](const V& v) { return v.rows; })
        .def_property_readonly("ghost_rows", [](const V&) { return 0; })
        .def_property_readonly("num_vectors", [](const V& v) { return v.k; });
  } else {
    cls.def("pointwise_mult", [](V& a, const V& b) { a.pointwise(b, false); })
        .def("dot", [](const V& a, const V& b) { return a.bdot(b)[0]; })
        .def_property_readonly("local_size", [](const V& v) { return v.rows; })
        .def_property_readonly("ghost_size", [](const V&) { return 0; })
        .def_property_readonly("full_size", [](const V& v) { return v.rows; });
  }
}

template <typename T>
void bind_matrix(py::module& m, const char* name) {
  using M = Mat<T>;
  using MV = DV<T, true>;
  using SV = DV<T, false>;
  auto unsupported = [](const char* what) {
    return std::string(what) + " is not available in the single-GPU B200 engine";
  };
  py::class_<M>(m, name)
      .def(py::init([](GraphPtr g) { return std::make_unique<M>(g); }), py::keep_alive<1, 2>())
      .def_property_readonly("graph", [](const M& a) { return a.g; })
      .def("add_block", &M::add_block, py::arg("g_row"), py::arg("g_col"), py::arg("data"),
           py::arg("mode") = AssemblyMode::ADD)
      .def("set_values", &M::set_values, py::arg("values"))
      .def("assemble", [](M&) {})
      .def("mult", [](M& a, SV& x, SV& y) { a.mult(x, y, false); })
      .def("mult_dense", [](M& a, MV& x, MV& y) { a.mult(x, y, false); })
      .def("mult_adjoint", [](M& a, SV& x, SV& y) { a.mult(x, y, true); })
      .def("mult_dense_adjoint", [](M& a, MV& x, MV& y) { a.mult(x, y, true); })
      .def("scale", [](M& a, T alpha) {
        a.ensure_device();
        const cplx z(alpha);
        check(vbg_matrix_scale(a.dm, z.real(), z.imag(), stream()), "scale");
        a.device_modified();
      })
      .def("shift", [](M& a, T alpha) {
        a.ensure_device();
        const cplx z(alpha);
        check(vbg_matrix_shift(a.dm, z.real(), z.imag(), stream()), "shift");
        a.device_modified();
      })
      .def("add_diagonal", [](M& a, SV& v) {
        if (v.rows < a.g->N()) throw std::runtime_error("Vector size too small for add_diagonal");
        a.ensure_device();
        check(vbg_matrix_add_diagonal(a.dm, v.read(), stream()), "add_diagonal");
        a.device_modified();
      })
      .def("conjugate", [](M& a) {
        a.ensure_device();
        check(vbg_matrix_conjugate(a.dm, stream()), "conjugate");
        a.device_modified();
      })
      .def("axpby", [](M& y, T alpha, M& x, T beta) {
        y.ensure_device();
        x.ensure_device();
        const cplx za(alpha), zb(beta);
        check(vbg_matrix_axpby(y.dm, za.real(), za.imag(), x.dm, zb.real(), zb.imag(), stream()), "axpby");
        y.adopt_device_structure();
      })
      .def("axpy", [](M& y, T alpha, M& x) {
        y.ensure_device();
        x.ensure_device();
        const cplx za(alpha);
        check(vbg_matrix_axpby(y.dm, za.real(), za.imag(), x.dm, 1.0, 0.0, stream()), "axpy");
        y.adopt_device_structure();
      })
      .def("copy_from", [](M& a, M& b) {
        if (a.g->row_ptr != b.g->row_ptr || a.g->col_ind != b.g->col_ind || a.g->bsz != b.g->bsz)
          throw std::runtime_error("Incompatible graph structure in copy_from");
        b.ensure_host();
        a.host = b.host;
        a.host_ok = true;
        a.host_modified();
      })
      .def("fill", [](M& a, T v) {
        a.ensure_host();
        std::fill(a.host.begin(), a.host.end(), v);
        a.host_modified();
      })
      .def("fill_random", [](M& a) {
        // uniform [0, 1) from a fixed-seed splitmix64 counter (reproducible)
        a.ensure_host();
        uint64_t x = 0;
        for (auto& v : a.host) {
          x += 0x9e3779b97f4a7c15ULL;
          uint64_t z = x;
          z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
          z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
          z ^= z >> 31;
          v = T((double)(z >> 11) * (1.0 / 9007199254740992.0));
        }
        a.host_modified();
      })
      .def("duplicate", [](M& a, bool independent_graph) {
        auto g = independent_graph ? std::make_shared<Graph>(*a.g) : a.g;
        auto d = std::make_unique<M>(g, 0);
        if (a.dev_ok && a.dm) {
          check(vbg_matrix_duplicate(a.dm, &d->dm, stream()), "duplicate");
          d->dev_ok = true;
          d->host_ok = false;
        } else {
          d->host = a.host;
          d->host_ok = true;
        }
        return d;
      }, py::arg("independent_graph") = true)
      .def("spmm", [](M& a, M& b, double thr, bool transA, bool transB) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix *at = nullptr, *bt = nullptr, *c = nullptr;
        if (transA) check(vbg_matrix_transpose(a.dm, &at, stream()), "transpose");
        if (transB) check(vbg_matrix_transpose(b.dm, &bt, stream()), "transpose");
        const int rc = vbg_spgemm(at ? at : a.dm, bt ? bt : b.dm, thr, &c, nullptr, stream());
        if (at) vbg_matrix_destroy(at);
        if (bt) vbg_matrix_destroy(bt);
        check(rc, "spmm");
        return M::wrap_device(c);
      }, py::arg("B"), py::arg("threshold"), py::arg("transA") = false, py::arg("transB") = false)
      .def("spmm_self", [](M& a, double thr, bool transA) {
        a.ensure_device();
        vbg_matrix *at = nullptr, *c = nullptr;
        if (transA) check(vbg_matrix_transpose(a.dm, &at, stream()), "transpose");
        const int rc = vbg_spgemm(at ? at : a.dm, at ? at : a.dm, thr, &c, nullptr, stream());
        if (at) vbg_matrix_destroy(at);
        check(rc, "spmm_self");
        return M::wrap_device(c);
      }, py::arg("threshold"), py::arg("transA") = false)
      .def("spmm_hermitian", [](M& a, M& b, double thr, bool transA) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix *at = nullptr, *c = nullptr;
        if (transA) check(vbg_matrix_transpose(a.dm, &at, stream()), "transpose");
        const int rc = vbg_spgemm_hermitian(at ? at : a.dm, b.dm, thr, &c, nullptr, stream());
        if (at) vbg_matrix_destroy(at);
        check(rc, "spmm_hermitian");
        return M::wrap_device(c);
      }, py::arg("B"), py::arg("threshold"), py::arg("transA") = false)
      .def("add", [](M& a, M& b, double alpha, double beta) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix* d = nullptr;
        check(vbg_matrix_duplicate(a.dm, &d, stream()), "duplicate");
        auto c = M::wrap_device(d);
        check(vbg_matrix_scale(c->dm, alpha, 0.0, stream()), "scale");
        check(vbg_matrix_axpby(c->dm, beta, 0.0, b.dm, 1.0, 0.0, stream()), "axpy");
        c->adopt_device_structure();
        return c;
      }, py::arg("B"), py::arg("alpha") = 1.0, py::arg("beta") = 1.0)
      .def("transpose", [](M& a) {
        a.ensure_device();
        vbg_matrix* t = nullptr;
        check(vbg_matrix_transpose(a.dm, &t, stream()), "transpose");
        return M::wrap_device(t);
      })
      .def("real", [](M& a) {
        a.ensure_host();
        auto r = std::make_unique<MatD>(a.g);
        for (size_t i = 0; i < a.host.size(); ++i) r->host[i] = cplx(a.host[i]).real();
        r->host_modified();
        return r;
      })
      .def("imag", [](M& a) {
        a.ensure_host();
        auto r = std::make_unique<MatD>(a.g);
        for (size_t i = 0; i < a.host.size(); ++i) r->host[i] = cplx(a.host[i]).imag();
        r->host_modified();
        return r;
      })
      .def("filter_blocks", [](M& a, double thr) {
        if (thr <= 0.0) return;
        a.ensure_device();
        check(vbg_matrix_filter_blocks(a.dm, thr, stream()), "filter_blocks");
        a.adopt_device_structure();
      })
      .def("get_block_density", [](const M& a) {
        const double n = a.g->n;
        return n == 0 ? 0.0 : (double)a.g->nnzb() / (n * n);
      })
      .def("get_block", [](M& a, int row, int col) {
        if (row < 0 || row >= a.g->n || col < 0 || col >= a.g->n) return py::array_t<T>();
        const int s = a.g->slot(row, col);
        if (s < 0) return py::array_t<T>();
        a.ensure_host();
        const int rd = a.g->bsz[row], cd = a.g->bsz[col];
        py::array_t<T> out({rd, cd});
        std::memcpy(out.mutable_data(), a.host.data() + a.g->slot_offsets()[s], sizeof(T) * rd * cd);
        return out;
      }, py::arg("row"), py::arg("col"))
      .def("get_values", [](M& a) {
        a.ensure_host();
        return to_array(a.host);
      })
      .def("to_dense", [](M& a) {
        a.ensure_host();
        const int64_t N = a.g->N();
        py::array_t<T> out({N, N});
        T* d = out.mutable_data();
        std::fill(d, d + N * N, T(0));
        const auto off = a.g->slot_offsets();
        for (int i = 0; i < a.g->n; ++i)
          for (int s = a.g->row_ptr[i]; s < a.g->row_ptr[i + 1]; ++s) {
            const int j = a.g->col_ind[s], rd = a.g->bsz[i], cd = a.g->bsz[j];
            for (int t = 0; t < rd; ++t)
              for (int q = 0; q < cd; ++q)
                d[(a.g->scal_off[i] + t) * N + a.g->scal_off[j] + q] += a.host[off[s] + t * cd + q];
          }
        return out;
      })
      .def("from_dense", [](M& a, py::array_t<T, py::array::c_style | py::array::forcecast> arr) {
        const int64_t N = a.g->N();
        if (arr.ndim() != 2 || arr.shape(0) != N || arr.shape(1) != N)
          throw std::runtime_error("from_dense: expected shape (" + std::to_string(N) + ", " + std::to_string(N) + ")");
        a.ensure_host();
        const T* d = arr.data();
        const auto off = a.g->slot_offsets();
        for (int i = 0; i < a.g->n; ++i)
          for (int s = a.g->row_ptr[i]; s < a.g->row_ptr[i + 1]; ++s) {
            const int j = a.g->col_ind[s], rd = a.g->bsz[i], cd = a.g->bsz[j];
            for (int t = 0; t < rd; ++t)
              for (int q = 0; q < cd; ++q)
                a.host[off[s] + t * cd + q] = d[(a.g->scal_off[i] + t) * N + a.g->scal_off[j] + q];
          }
        a.host_modified();
      }, py::arg("array"))
      .def("save_matrix_market", [](M& a, const std::string& fn) {
        a.ensure_host();
        std::ofstream f(fn);
        if (!f) throw std::runtime_error("save_matrix_market: cannot open " + fn);
        const bool z = dtype_code<T>() == VBG_C128;
        f << "%%MatrixMarket matrix coordinate " << (z ? "complex" : "real") << " general\n";
        const int64_t N = a.g->N();
        f << N << " " << N << " " << a.host.size() << "\n" << std::setprecision(17);
        const auto off = a.g->slot_offsets();
        for (int i = 0; i < a.g->n; ++i)
          for (int s = a.g->row_ptr[i]; s < a.g->row_ptr[i + 1]; ++s) {
            const int j = a.g->col_ind[s], rd = a.g->bsz[i], cd = a.g->bsz[j];
            for (int t = 0; t < rd; ++t)
              for (int q = 0; q < cd; ++q) {
                const cplx v(a.host[off[s] + t * cd + q]);
                f << a.g->scal_off[i] + t + 1 << " " << a.g->scal_off[j] + q + 1 << " " << v.real();
                if (z) f << " " << v.imag();
                f << "\n";
              }
          }
      })
      .def("extract_submatrix", [unsupported](M&, std::vector<int>) -> std::unique_ptr<M> {
        throw std::runtime_error(unsupported("extract_submatrix"));
      })
      .def("insert_submatrix", [unsupported](M&, M&, std::vector<int>) {
        throw std::runtime_error(unsupported("insert_submatrix"));
      })
      .def("spmf", [unsupported](M&, std::string, bool) -> std::unique_ptr<M> {
        throw std::runtime_error(unsupported("spmf (graph matrix functions)"));
      }, py::arg("func_name"), py::arg("verbose") = false)
      .def("redistribute", [unsupported](M&, GraphPtr, AssemblyMode) -> std::unique_ptr<M> {
        throw std::runtime_error(unsupported("redistribute (MPI ranks)"));
      }, py::arg("target_graph"), py::arg("mode") = AssemblyMode::INSERT)
      // vbcsr/pybind_vbcsr.cpp binds redistribute_cross(target_graph, op,
      // common_comm) for moving a matrix between communicators; one rank here
      .def("redistribute_cross", [unsupported](M&, py::object, RedistOp, py::object) -> std::unique_ptr<M> {
        throw std::runtime_error(unsupported("redistribute_cross (MPI communicators)"));
      }, py::arg("target_graph"), py::arg("op") = RedistOp::Copy, py::arg("common_comm") = py::none())
      .def_property_readonly("matrix_kind", [](const M& a) {
        int mn = INT32_MAX, mx = 0;
        for (int b : a.g->bsz) {
          mn = std::min(mn, b);
          mx = std::max(mx, b);
        }
        return std::string(mx <= 1 ? "csr" : (mn == mx ? "bsr" : "vbcsr"));
      })
      .def_property_readonly("local_nnz", [](const M& a) { return a.g->nnz(); })
      .def_property_readonly("global_nnz", [](const M& a) { return a.g->nnz(); })
      .def_property_readonly("local_block_nnz", [](const M& a) { return a.g->nnzb(); })
      .def_property_readonly("owned_scalar_rows", [](const M& a) { return a.g->N(); })
      .def_property_readonly("global_scalar_rows", [](const M& a) { return a.g->N(); })
      .def_property_readonly("global_scalar_cols", [](const M& a) { return a.g->N(); })
      .def_property_readonly("shape", [](const M& a) { return py::make_tuple(a.g->N(), a.g->N()); })
      .def_property_readonly("row_ptr", [](const M& a) { return to_array(a.g->row_ptr); })
      .def_property_readonly("col_ind", [](const M& a) { return to_array(a.g->col_ind); })
      .def_property_readonly("configured_page_size", [](const M&) { return 0; })
      .def_property("page_size", [](const M&) { return 0; }, [](M&, uint32_t) {})
      .def("set_page_size", [](M&, uint32_t) {}, py::arg("page_size"))
      .def_property_readonly("shape_class_count", [](const M& a) {
        std::vector<std::pair<int, int>> shapes;
        for (int i = 0; i < a.g->n; ++i)
          for (int s = a.g->row_ptr[i]; s < a.g->row_ptr[i + 1]; ++s)
            shapes.emplace_back(a.g->bsz[i], a.g->bsz[a.g->col_ind[s]]);
        std::sort(shapes.begin(), shapes.end());
        return (int)(std::unique(shapes.begin(), shapes.end()) - shapes.begin());
      })
      .def_property_readonly("vendor_backend_name", [](const M&) { return std::string("b200"); })
      .def_property_readonly("vendor_launch_count", [](const M&) { return 0; })
      .def("reset_vendor_launch_count", [](M&) {})
      .def_property_readonly("has_contiguous_layout", [](const M&) { return true; })
      .def("pack_contiguous", [](M&) {})
      // ---- engine extensions (not in the reference) ----
      .def("spmm_ex", [](M& a, M& b, double thr, int precision, bool hermitian) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix* c = nullptr;
        check(vbg_spgemm_ex(a.dm, b.dm, thr, precision, hermitian ? 1 : 0, &c, nullptr, stream()), "spmm_ex");
        return M::wrap_device(c);
      }, py::arg("B"), py::arg("threshold"), py::arg("precision") = 0, py::arg("hermitian") = false)
      // the reference core's fused triple products (BlockSpMat methods in
      // block_csr.hpp:1804-1853, not bound to Python there): upper triangle
      .def("square_polynomial_upper", [](M& a, cplx c2, cplx c1, cplx c0, double thr) {
        a.ensure_device();
        vbg_matrix* c = nullptr;
        check(vbg_square_polynomial_upper(a.dm, c2.real(), c2.imag(), c1.real(), c1.imag(), c0.real(), c0.imag(),
                                          thr, &c, stream()),
              "square_polynomial_upper");
        return M::wrap_device(c);
      }, py::arg("c2"), py::arg("c1"), py::arg("c0"), py::arg("threshold"))
      .def("rarh_upper", [](M& a, M& b, double thr) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix* c = nullptr;
        check(vbg_rarh_upper(a.dm, b.dm, thr, &c, stream()), "rarh_upper");
        return M::wrap_device(c);
      }, py::arg("B"), py::arg("threshold"))
      .def("rhar_upper", [](M& a, M& b, double thr) {
        a.ensure_device();
        b.ensure_device();
        vbg_matrix* c = nullptr;
        check(vbg_rhar_upper(a.dm, b.dm, thr, &c, stream()), "rhar_upper");
        return M::wrap_device(c);
      }, py::arg("B"), py::arg("threshold"))
      .def("complete_hermitian", [](M& a) {
        a.ensure_device();
        vbg_matrix* d = nullptr;
        check(vbg_matrix_duplicate(a.dm, &d, stream()), "duplicate");
        auto c = M::wrap_device(d);
        check(vbg_matrix_complete_hermitian(c->dm, stream()), "complete_hermitian");
        c->adopt_device_structure();
        return c;
      })
      .def("complete_hermitian_inplace", [](M& a) {
        a.ensure_device();
        check(vbg_matrix_complete_hermitian(a.dm, stream()), "complete_hermitian");
        a.adopt_device_structure();
      })
      .def("trace_fp64", [](M& a) {
        a.ensure_device();
        DBuf d;
        d.ensure(16);
        check(vbg_matrix_trace(a.dm, static_cast<double*>(d.p), stream()), "trace");
        double h[2] = {0.0, 0.0};
        cuda_check(cudaMemcpyAsync(h, d.p, 16, cudaMemcpyDeviceToHost, stream()), "D2H");
        cuda_check(cudaStreamSynchronize(stream()), "sync");
        return cplx(h[0], h[1]);
      })
      .def("norm_fro_fp64", [](M& a) {
        a.ensure_device();
        DBuf d;
        d.ensure(16);
        check(vbg_matrix_norm_fro(a.dm, static_cast<double*>(d.p), stream()), "norm_fro");
        double h[2] = {0.0, 0.0};
        cuda_check(cudaMemcpyAsync(h, d.p, 16, cudaMemcpyDeviceToHost, stream()), "D2H");
        cuda_check(cudaStreamSynchronize(stream()), "sync");
        return h[0];
      })
      .def("kpm_moments", [](M& a, MV& v0, int nmom, int precision, bool two_moment, bool use_graph) {
        a.ensure_device();
        DBuf mu;
        mu.ensure((size_t)nmom * 8);
        check(vbg_kpm_moments(a.dm, v0.k, v0.ld, v0.read(), nmom, precision, two_moment ? 1 : 0, use_graph ? 1 : 0,
                              static_cast<double*>(mu.p), stream()),
              "kpm_moments");
        std::vector<double> out(nmom);
        cuda_check(cudaMemcpyAsync(out.data(), mu.p, nmom * 8, cudaMemcpyDeviceToHost, stream()), "D2H");
        cuda_check(cudaStreamSynchronize(stream()), "sync");
        return to_array(out);
      }, py::arg("v0"), py::arg("num_moments"), py::arg("precision") = 0, py::arg("two_moment") = true,
         py::arg("use_graph") = true)
      .def("cheb_step", [](M& a, py::object xo, py::object xprev, py::object yo, double alpha, double beta,
                           double gamma, py::object dot_with, bool want_dots, py::object acc, cplx coef) {
        a.ensure_device();
        Vec<T>& x = vec_of<T>(xo);
        Vec<T>& y = vec_of<T>(yo);
        if (!a.g->same_owned_structure(*x.g) || !a.g->same_owned_structure(*y.g))
          throw std::runtime_error("cheb_step: graph mismatch");
        const void* xp = x.read();
        const void* pp = xprev.is_none() ? nullptr : vec_of<T>(xprev).read();
        const void* dw = dot_with.is_none() ? nullptr : vec_of<T>(dot_with).read();
        void* ap = acc.is_none() ? nullptr : vec_of<T>(acc).readwrite();
        void* yp = y.write_all();
        DBuf dd;
        double* dots = nullptr;
        if (want_dots) {
          dd.ensure(16);
          dots = static_cast<double*>(dd.p);
        }
        check(vbg_cheb_step(a.dm, x.k, x.ld, alpha, beta, gamma, xp, pp, yp, dw, dots, ap, coef.real(), coef.imag(),
                            stream()),
              "cheb_step");
        std::vector<double> h(2, 0.0);
        if (want_dots) {
          cuda_check(cudaMemcpyAsync(h.data(), dots, 16, cudaMemcpyDeviceToHost, stream()), "D2H");
          cuda_check(cudaStreamSynchronize(stream()), "sync");
        }
        return py::make_tuple(h[0], h[1]);
      }, py::arg("x"), py::arg("xprev"), py::arg("y"), py::arg("alpha"), py::arg("beta"), py::arg("gamma"),
         py::arg("dot_with") = py::none(), py::arg("want_dots") = false, py::arg("acc") = py::none(),
         py::arg("acc_coef") = cplx(0.0, 0.0))
      .def("cheb_series", [](M& a, py::object vo, py::array_t<cplx, py::array::c_style | py::array::forcecast> coeffs,
                             double scale, double center, py::object yo) {
        // y = sum_n c_n T_n((A - center) / scale) v, all terms in one library call
        a.ensure_device();
        Vec<T>& v = vec_of<T>(vo);
        Vec<T>& y = vec_of<T>(yo);
        if (!a.g->same_owned_structure(*v.g) || !a.g->same_owned_structure(*y.g))
          throw std::runtime_error("cheb_series: graph mismatch");
        if (v.k != y.k || v.ld != y.ld) throw std::runtime_error("cheb_series: vector shape mismatch");
        const py::ssize_t n = coeffs.size();
        if (n < 1 || n > INT32_MAX) throw std::runtime_error("cheb_series: need 1 .. 2^31-1 coefficients");
        std::vector<double> c(2 * (size_t)n);
        const cplx* cp = coeffs.data();
        for (py::ssize_t i = 0; i < n; ++i) {
          c[2 * i] = cp[i].real();
          c[2 * i + 1] = cp[i].imag();
        }
        const void* vp = v.read();
        void* yp = y.write_all();
        check(vbg_cheb_series(a.dm, v.k, v.ld, vp, (int)n, c.data(), scale, center, yp, 0, nullptr, stream()),
              "cheb_series");
      }, py::arg("v"), py::arg("coeffs"), py::arg("scale"), py::arg("center"), py::arg("y"));
}

}  // namespace

PYBIND11_MODULE(vbcsr_core, m) {
  m.doc() = "VBCSR core on the B200 engine (serial, one GPU)";
  m.def("threading_diagnostics", [](bool) {
    py::dict d;
    d["openmp_enabled"] = false;
    d["omp_get_max_threads"] = 1;
    d["mkl_enabled"] = false;
    d["mkl_get_max_threads_before"] = py::none();
    d["mkl_get_max_threads_after"] = py::none();
    d["cuda_devices"] = vbg_device_count();
    return d;
  }, py::arg("configure_vendor_sparse") = false);
  py::enum_<AssemblyMode>(m, "AssemblyMode")
      .value("INSERT", AssemblyMode::INSERT)
      .value("ADD", AssemblyMode::ADD)
      .export_values();
  py::enum_<RedistOp>(m, "RedistOp").value("Copy", RedistOp::Copy).value("Sum", RedistOp::Sum).export_values();
  m.def("finalize_mpi", []() {});

  // The atomic-structure surface of the reference (vbcsr/pybind_atomic.cpp:
  // AtomicData :208, the PhaseConvention enum :482-485, ImageContainer /
  // ImageContainer_Complex :78,487-488) is not part of this engine.  The
  // names exist so that the reference's package imports unchanged on top of
  // this module (vbcsr/atomic_data.py:30 subclasses AtomicData,
  // vbcsr/image_container.py:2 imports PhaseConvention); constructing any of
  // them raises.
  py::enum_<PhaseConvention>(m, "PhaseConvention")
      .value("R_ONLY", PhaseConvention::R_ONLY)
      .value("R_AND_POSITION", PhaseConvention::R_AND_POSITION)
      .export_values();
  py::class_<AtomicDataStub>(m, "AtomicData")
      .def(py::init([](py::args, py::kwargs) -> AtomicDataStub* {
        throw std::runtime_error("AtomicData (atomic structures, neighbour lists) is not available in the B200 engine");
      }));
  py::class_<ImageContainerStub>(m, "ImageContainer")
      .def(py::init([](py::args, py::kwargs) -> ImageContainerStub* {
        throw std::runtime_error("ImageContainer (periodic images, k-sampling) is not available in the B200 engine");
      }));
  py::class_<ImageContainerComplexStub>(m, "ImageContainer_Complex")
      .def(py::init([](py::args, py::kwargs) -> ImageContainerComplexStub* {
        throw std::runtime_error("ImageContainer (periodic images, k-sampling) is not available in the B200 engine");
      }));

  py::class_<Graph, GraphPtr>(m, "DistGraph")
      .def(py::init([](py::object comm) {
             if (!comm.is_none() && py::hasattr(comm, "Get_size") && comm.attr("Get_size")().cast<int>() > 1)
               throw std::runtime_error("vbcsr_core (B200): communicators with more than one rank are not supported");
             return std::make_shared<Graph>();
           }),
           py::arg("comm") = py::none())
      .def("construct_serial", [](Graph& g, int n, std::vector<int> sizes, std::vector<std::vector<int>> adj) {
        if ((int)sizes.size() != n)
          throw std::runtime_error("DistGraph::construct_serial received invalid block size metadata on root");
        if ((int)adj.size() != n)
          throw std::runtime_error("DistGraph::construct_serial received invalid adjacency metadata on root");
        g.set_lists(n, sizes, adj);
      })
      .def("construct_distributed", [](Graph& g, std::vector<int> owned, std::vector<int> sizes,
                                       std::vector<std::vector<int>> adj) {
        if (!std::is_sorted(owned.begin(), owned.end()))
          throw std::runtime_error("DistGraph::construct_distributed requires sorted owned_global_indices");
        for (size_t i = 0; i < owned.size(); ++i)
          if (owned[i] != (int)i)
            throw std::runtime_error("vbcsr_core (B200): distributed graphs are not supported; owned indices must be 0..n-1");
        g.set_lists((int)owned.size(), sizes, adj);
      })
      .def("construct_distributed_flat",
           [](Graph& g, py::array_t<int, py::array::c_style | py::array::forcecast> owned,
              py::array_t<int, py::array::c_style | py::array::forcecast> sizes,
              py::array_t<int64_t, py::array::c_style | py::array::forcecast> aptr,
              py::array_t<int, py::array::c_style | py::array::forcecast> aind) {
             const py::ssize_t n = owned.shape(0);
             if (sizes.shape(0) != n || aptr.shape(0) != n + 1)
               throw std::runtime_error(
                   "construct_distributed_flat: block_sizes must match owned_indices and adj_ptr must have one more "
                   "entry than owned_indices");
             for (py::ssize_t i = 0; i < n; ++i)
               if (owned.data()[i] != (int)i)
                 throw std::runtime_error(
                     "vbcsr_core (B200): distributed graphs are not supported; owned indices must be 0..n-1");
             std::vector<int> sv(sizes.data(), sizes.data() + n);
             g.set_rows((int)n, sv, aptr.data(), aind.data());
           },
           py::arg("owned_indices"), py::arg("block_sizes"), py::arg("adj_ptr"), py::arg("adj_ind"))
      .def_property_readonly("owned_global_indices", [](const Graph& g) {
        std::vector<int> v(g.n);
        std::iota(v.begin(), v.end(), 0);
        return v;
      })
      .def_property_readonly("ghost_global_indices", [](const Graph&) { return std::vector<int>(); })
      .def_property_readonly("block_sizes", [](const Graph& g) { return g.bsz; })
      .def_property_readonly("adj_ptr", [](const Graph& g) { return g.row_ptr; })
      .def_property_readonly("adj_ind", [](const Graph& g) { return g.col_ind; })
      .def_property_readonly("owned_scalar_rows", [](const Graph& g) { return g.N(); })
      .def_property_readonly("local_scalar_cols", [](const Graph& g) { return g.N(); })
      .def_property_readonly("global_scalar_rows", [](const Graph& g) { return g.N(); })
      .def("get_local_index", [](const Graph& g, int gid) { return (gid >= 0 && gid < g.n) ? gid : -1; })
      .def("get_global_index", [](const Graph& g, int lid) { return (lid >= 0 && lid < g.n) ? lid : -1; })
      .def_property_readonly("rank", [](const Graph&) { return 0; })
      .def_property_readonly("size", [](const Graph&) { return 1; });

  bind_vector<double, false>(m, "DistVector_Double");
  bind_vector<cplx, false>(m, "DistVector_Complex");
  bind_vector<double, true>(m, "DistMultiVector_Double");
  bind_vector<cplx, true>(m, "DistMultiVector_Complex");
  bind_matrix<double>(m, "BlockSpMat_Double");
  bind_matrix<cplx>(m, "BlockSpMat_Complex");
}
