// pybind11 module `hignn`: the reference's Python interface over the C ABI.
//
// Mirrors interface/HignnInterface.cpp:9-92 -- Init/Finalize, HignnModel with
// the same method names and argument meaning, ExplicitEuler and ExplicitRk4
// (include/TimeIntegrator.hpp:424-861) -- so a script written for the
// reference runs unchanged:
//     import hignn; m = hignn.HignnModel(X, 128); m.load_two_body_model(p)
//     m.update_coord(X); m.dot(u, f)
// Differences, all of them failing loudly where the reference fails silently
// or aborts: arrays are shape-checked; `u` must be a writable C-contiguous
// float32 (n, 3) array (the reference force-casts other dtypes into a
// temporary and the result is lost); status codes of the C ABI become
// RuntimeError. The GIL is released around device work.
#include <pybind11/functional.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "hignn_b200.h"

namespace py = pybind11;

namespace {

void check(int st) {
  if (st != HIGNN_OK) {
    char buf[2048];
    hignn_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string("hignn: ") + buf);
  }
}

using farr = py::array_t<float, py::array::c_style | py::array::forcecast>;

farr as_n3(const py::array& a, const char* what) {
  farr v = farr::ensure(a);
  if (!v || v.ndim() != 2 || v.shape(1) < 3) throw std::invalid_argument(std::string(what) + " must be (n, 3) float");
  if (v.shape(1) != 3) {
    // positions passed as (n, 6) [x, y, z, angles] are accepted, as the reference reads columns 0..2
    farr out({v.shape(0), (py::ssize_t)3});
    auto s = v.unchecked<2>();
    auto d = out.mutable_unchecked<2>();
    for (py::ssize_t i = 0; i < v.shape(0); i++)
      for (int k = 0; k < 3; k++) d(i, k) = s(i, k);
    return out;
  }
  return v;
}

int default_device() {
  const char* lr = std::getenv("LOCAL_RANK");
  int rank = lr ? std::atoi(lr) : 0;
  return rank;  // the C ABI checks it against the device count
}

class HignnModel {
 public:
  HignnModel(py::array coord, int blockSize) {
    farr x = as_n3(coord, "coord");
    n_ = x.shape(0);
    check(hignn_create(x.data(), n_, blockSize, default_device(), &m_));
  }
  ~HignnModel() {
    if (m_) hignn_destroy(m_);
  }
  void load_two_body_model(const std::string& path) {
    // the reference appends "_<dev>.pt"; here the base path resolves to an .hgnw blob
    std::string p = py::module_::import("hignn_b200.weights").attr("resolve_model_path")(path).cast<std::string>();
    check(hignn_load_two_body(m_, p.c_str()));
  }
  void load_three_body_model(const std::string&) {}  // a no-op in the reference (src/HignnModel.cpp:444-446)
  void set(int key, double v) { check(hignn_set_param(m_, key, v)); }
  double get(int key) {
    double v = 0;
    check(hignn_get_param(m_, key, &v));
    return v;
  }
  void update_coord(py::array coord) {
    farr x = as_n3(coord, "coord");
    if (x.shape(0) != n_) throw std::invalid_argument("update_coord: particle count changed");
    const float* p = x.data();
    py::gil_scoped_release nogil;
    check(hignn_update_coord(m_, p, n_));
  }
  // addition: new positions on the kept tree (a simulation that rebuilds every k steps)
  void update_coord_keep_tree(py::array coord) {
    farr x = as_n3(coord, "coord");
    if (x.shape(0) != n_) throw std::invalid_argument("update_coord_keep_tree: particle count changed");
    const float* p = x.data();
    py::gil_scoped_release nogil;
    check(hignn_update_coord_keep_tree(m_, p, n_));
  }
  void dot(py::array uArray, py::array fArray) { run(uArray, fArray, false); }
  void dense_dot(py::array uArray, py::array fArray) { run(uArray, fArray, true); }
  py::dict stats() {
    hignn_stats s{};
    check(hignn_get_stats(m_, &s));
    py::dict d;
    d["n"] = s.n;
    d["num_nodes"] = s.num_nodes;
    d["num_leaves"] = s.num_leaves;
    d["num_close"] = s.num_close;
    d["num_far"] = s.num_far;
    d["close_evals"] = s.close_evals;
    d["far_evals"] = s.far_evals;
    d["far_rank_sum"] = s.far_rank_sum;
    d["far_rank_max"] = s.far_rank_max;
    d["t_build_ms"] = s.t_build_ms;
    d["t_close_ms"] = s.t_close_ms;
    d["t_far_ms"] = s.t_far_ms;
    d["t_dot_ms"] = s.t_dot_ms;
    return d;
  }

 private:
  void run(py::array uArray, py::array fArray, bool dense) {
    farr f = as_n3(fArray, "f");
    if (f.shape(0) != n_) throw std::invalid_argument("f has the wrong number of rows");
    auto u = py::array_t<float>::ensure(uArray);
    if (!uArray.dtype().is(py::dtype::of<float>()) || !(uArray.flags() & py::array::c_style) || !uArray.writeable() ||
        uArray.ndim() != 2 || uArray.shape(0) != n_ || uArray.shape(1) != 3)
      throw std::invalid_argument("u must be a writable C-contiguous float32 array of shape (n, 3)");
    float* up = static_cast<float*>(uArray.mutable_data());
    const float* fp = f.data();
    py::gil_scoped_release nogil;
    check(dense ? hignn_dense_dot(m_, up, fp, n_) : hignn_dot(m_, up, fp, n_));
  }
  hignn_model* m_ = nullptr;
  int64_t n_ = 0;
};

// ------------------------------------------------------------- time integration
// include/TimeIntegrator.hpp:39-409 (TimeIntegrator), :424-489 (ExplicitEuler),
// :500-861 (ExplicitRk4, adaptive Dormand-Prince 5(4)). Positions are float;
// t and dt are double. Angular velocities are never produced by the velocity
// callback (the reference leaves them at zero), so orientations stay at their
// initial Euler angles and are passed through unchanged. Without an output
// function nothing is written (the reference falls back to VTK files).
class TimeIntegrator {
 public:
  virtual ~TimeIntegrator() = default;
  void set_time_step(float v) { dt0_ = v; }
  void set_final_time(float v) { tf_ = v; }
  void set_num_rigid_body(size_t n) {
    n_ = n;
    x_.assign(3 * n, 0.f);
    ang_.assign(3 * n, 0.f);
    v_.assign(3 * n, 0.f);
    off_.assign(3 * n, 0.f);
  }
  void set_velocity_func(std::function<py::array_t<float>(float, py::array_t<float>)> f) { vel_ = std::move(f); }
  void set_output_func(std::function<void(py::array_t<float>, py::array_t<float>)> f) {
    out_ = std::move(f);
    custom_out_ = true;
  }
  void set_lim(int d, py::list lim) {
    lo_[d] = lim[0].cast<float>();
    hi_[d] = lim[1].cast<float>();
    periodic_ = true;
  }
  void set_output_step(int s) { out_step_ = s > 0 ? s : 1; }
  void initialize(py::array a) {
    auto p = farr::ensure(a);
    if (!p || p.ndim() != 2) throw std::runtime_error("Number of dimensions of input positions must be two");
    if ((size_t)p.shape(0) != n_) throw std::runtime_error("Inconsistent number of rigid bodies");
    if (p.shape(1) < 3) throw std::runtime_error("positions need at least 3 columns");
    auto s = p.unchecked<2>();
    for (size_t i = 0; i < n_; i++) {
      for (int k = 0; k < 3; k++) x_[3 * i + k] = s(i, k);
      for (int k = 0; k < 3; k++) ang_[3 * i + k] = p.shape(1) >= 6 ? s(i, 3 + k) : 0.f;
    }
  }
  int get_func_count() const { return count_; }

 protected:
  // VelocityUpdate (include/TimeIntegrator.hpp:92-141)
  void velocity(double t, const std::vector<float>& pos, std::vector<float>& vel) {
    py::array_t<float> in({(py::ssize_t)n_, (py::ssize_t)6});
    auto d = in.mutable_unchecked<2>();
    for (size_t i = 0; i < n_; i++) {
      for (int k = 0; k < 3; k++) {
        float o = 0.f;
        if (periodic_) {
          if (pos[3 * i + k] > hi_[k])
            o = lo_[k] - hi_[k];
          else if (pos[3 * i + k] < lo_[k])
            o = hi_[k] - lo_[k];
          off_[3 * i + k] = o;
        }
        d(i, k) = pos[3 * i + k] + o;
      }
      for (int k = 0; k < 3; k++) d(i, 3 + k) = ang_[3 * i + k];
    }
    if (!vel_) throw std::runtime_error("no velocity function set");
    py::array_t<float> r = vel_((float)t, in);
    auto rv = farr::ensure(r);
    if (!rv || rv.ndim() != 2 || (size_t)rv.shape(0) != n_ || rv.shape(1) < 3)
      throw std::runtime_error("velocity function must return an (n, 3) array");
    auto s = rv.unchecked<2>();
    for (size_t i = 0; i < n_; i++)
      for (int k = 0; k < 3; k++) vel[3 * i + k] = s(i, k);
  }
  void output() {
    if (!custom_out_) return;
    py::array_t<float> p({(py::ssize_t)n_, (py::ssize_t)3}), v({(py::ssize_t)n_, (py::ssize_t)3});
    std::copy(x_.begin(), x_.end(), p.mutable_data());
    std::copy(v_.begin(), v_.end(), v.mutable_data());
    out_(p, v);
  }
  void wrap_offsets() {
    if (!periodic_) return;
    for (size_t i = 0; i < n_; i++)
      for (int k = 0; k < 3; k++) {
        const float p = x_[3 * i + k];
        off_[3 * i + k] = p > hi_[k] ? lo_[k] - hi_[k] : (p < lo_[k] ? hi_[k] - lo_[k] : 0.f);
      }
  }
  size_t n_ = 0;
  double dt0_ = 1.0, tf_ = 10.0;
  int out_step_ = 1, count_ = 0;
  bool periodic_ = false, custom_out_ = false;
  float lo_[3] = {-1, -1, -1}, hi_[3] = {1, 1, 1};
  std::vector<float> x_, ang_, v_, off_;
  std::function<py::array_t<float>(float, py::array_t<float>)> vel_;
  std::function<void(py::array_t<float>, py::array_t<float>)> out_;
};

class ExplicitEuler : public TimeIntegrator {
 public:
  void run() {
    count_ = 0;
    double t = 0.0;
    const double h0 = dt0_;
    while (t < tf_ - 1e-5) {
      const double dt = std::min(h0, tf_ - t);
      velocity(t + dt, x_, v_);
      for (size_t q = 0; q < 3 * n_; q++) x_[q] = x_[q] + v_[q] * (float)dt;
      wrap_offsets();
      t += dt;
      if (count_ % out_step_ == 0) output();
      if (periodic_)
        for (size_t q = 0; q < 3 * n_; q++) x_[q] = x_[q] + off_[q];
      count_++;
    }
  }
};

class ExplicitRk4 : public TimeIntegrator {
 public:
  void set_threshold(double v) { thr_ = v; }
  void run() {
    // Dormand-Prince tableau (include/TimeIntegrator.hpp:503-549), float constants
    const float a21 = 1.f / 5.f;
    const float a31 = 3.f / 40.f, a32 = 9.f / 40.f;
    const float a41 = 44.f / 45.f, a42 = -56.f / 15.f, a43 = 32.f / 9.f;
    const float a51 = 19372.f / 6561.f, a52 = -25360.f / 2187.f, a53 = 64448.f / 6561.f, a54 = -212.f / 729.f;
    const float a61 = 9017.f / 3168.f, a62 = -355.f / 33.f, a63 = 46732.f / 5247.f, a64 = 49.f / 176.f,
                a65 = -5103.f / 18656.f;
    const float b1 = 35.f / 384.f, b3 = 500.f / 1113.f, b4 = 125.f / 192.f, b5 = -2187.f / 6784.f, b6 = 11.f / 84.f;
    const float dc1 = b1 - 5179.f / 57600.f, dc3 = b3 - 7571.f / 16695.f, dc4 = b4 - 393.f / 640.f,
                dc5 = b5 - (-92097.f) / 339200.f, dc6 = b6 - 187.f / 2100.f, dc7 = -1.f / 40.f;
    const float c[7] = {0.f, 1.f / 5.f, 3.f / 10.f, 4.f / 5.f, 8.f / 9.f, 1.f, 1.f};
    const size_t m = 3 * n_;
    std::vector<float> k[8];
    for (auto& v : k) v.assign(m, 0.f);  // k[1] stays zero before the first step, as in the reference
    std::vector<float> x0(m);
    count_ = 0;
    double t = 0.0;
    const double h0 = dt0_;
    velocity(t, x_, v_);  // writes the velocity, not k1 (include/TimeIntegrator.hpp:608)
    while (t < tf_ - 1e-5) {
      double dt = std::min(h0, tf_ - t);
      for (size_t q = 0; q < m; q++) x0[q] = periodic_ ? x_[q] + off_[q] : x_[q];
      double err = 100.0;
      while (err > thr_) {
        for (int i = 1; i < 7; i++) {
          for (size_t q = 0; q < m; q++) {
            float p = x0[q];
            switch (i) {
              case 1: p = p + k[1][q] * (float)(a21 * dt); break;
              case 2: p = p + k[1][q] * (float)(a31 * dt) + k[2][q] * (float)(a32 * dt); break;
              case 3:
                p = p + k[1][q] * (float)(a41 * dt) + k[2][q] * (float)(a42 * dt) + k[3][q] * (float)(a43 * dt);
                break;
              case 4:
                p = p + k[1][q] * (float)(a51 * dt) + k[2][q] * (float)(a52 * dt) + k[3][q] * (float)(a53 * dt) +
                    k[4][q] * (float)(a54 * dt);
                break;
              case 5:
                p = p + k[1][q] * (float)(a61 * dt) + k[2][q] * (float)(a62 * dt) + k[3][q] * (float)(a63 * dt) +
                    k[4][q] * (float)(a64 * dt) + k[5][q] * (float)(a65 * dt);
                break;
              case 6:
                p = p + k[1][q] * (float)(b1 * dt) + k[3][q] * (float)(b3 * dt) + k[4][q] * (float)(b4 * dt) +
                    k[5][q] * (float)(b5 * dt) + k[6][q] * (float)(b6 * dt);
                break;
            }
            x_[q] = p;
          }
          velocity(t + c[i] * dt, x_, v_);
          k[i + 1] = v_;
        }
        err = 0.0;
        for (size_t i = 0; i < n_; i++) {
          float ve[3];
          for (int d = 0; d < 3; d++) {
            const size_t q = 3 * i + d;
            ve[d] = (k[1][q] * dc1 + k[3][q] * dc3 + k[4][q] * dc4 + k[5][q] * dc5 + k[6][q] * dc6 +
                     k[7][q] * dc7) *
                    (float)dt;
          }
          err += (double)(ve[0] * ve[0] + ve[1] * ve[1] + ve[2] * ve[2]);  // Vec3::SquareMag is float
        }
        err = std::sqrt(err);
        if (err > thr_) {
          dt = dt * std::max(0.8 * std::pow(err / thr_, -0.2), 0.1);
          dt = std::max(dt, 1e-6);
        }
      }
      t += dt;
      const double temp = 1.25 * std::pow(err / thr_, 0.2);
      dt = temp > 0.2 ? dt / temp : dt * 5.0;
      dt = std::min(dt, h0);
      if (count_ % out_step_ == 0) output();
      k[1] = k[7];  // first-same-as-last
      count_++;
    }
  }

 private:
  double thr_ = 1e-3;
};

// PotentialForce (include/PotentialForce.hpp, bound at interface/HignnInterface.cpp:66-71):
// Morse pair forces of every particle from its neighbours within the two-body epsilon, here on
// the device (cell list) through hignn_pair_forces. The reference hard-codes De = 1, a = 1,
// re = 2.5; set_parameters changes them (an addition). Periodic images are not implemented:
// set_periodic(True) / set_domain raise.
class PotentialForce {
 public:
  PotentialForce() {
    const float origin[3] = {0.f, 0.f, 0.f};
    check(hignn_create(origin, 1, 128, default_device(), &m_));  // device context and buffers only
  }
  ~PotentialForce() {
    if (m_) hignn_destroy(m_);
  }
  void set_periodic(bool periodic) {
    if (periodic) throw std::runtime_error("hignn: periodic pair forces are not supported by hignn_b200");
  }
  void set_domain(py::array) {
    throw std::runtime_error("hignn: periodic pair forces are not supported by hignn_b200");
  }
  void set_two_body_epsilon(float eps) { eps_ = eps; }
  void set_parameters(double De, double a, double re) {
    De_ = De;
    a_ = a;
    re_ = re;
  }
  py::array_t<float> get_potential_force(py::array coord) {
    farr x = as_n3(coord, "coord");
    const int64_t n = x.shape(0);
    py::array_t<float> f({(py::ssize_t)n, (py::ssize_t)3});
    float* fp = f.mutable_data();
    const float* xp = x.data();
    {
      py::gil_scoped_release nogil;
      check(hignn_pair_forces(m_, xp, fp, n, nullptr, De_, a_, re_, eps_));
    }
    return f;
  }

 private:
  hignn_model* m_ = nullptr;
  double De_ = 1.0, a_ = 1.0, re_ = 2.5;
  float eps_ = 0.f;
};

// NeighborLists (include/NeighborLists.hpp, bound at interface/HignnInterface.cpp:73-91): the
// two-body, three-body and three-body self edge lists, built on the device. Getters return
// uint64 (rows, E) arrays as the reference's size_t arrays; each particle's neighbours are in
// ascending order (the reference's follow its kd-tree). Periodic images are not implemented in
// the reference either (its periodic branch builds no source sites): set_periodic(True) and
// set_domain raise.
class NeighborLists {
 public:
  NeighborLists() { check(hignn_nbl_create(default_device(), &l_)); }
  ~NeighborLists() {
    if (l_) hignn_nbl_destroy(l_);
  }
  void set_periodic(bool periodic) {
    if (periodic) throw std::runtime_error("hignn: periodic neighbour lists are not supported");
  }
  void set_domain(py::array) { throw std::runtime_error("hignn: periodic neighbour lists are not supported"); }
  void update_coord(py::array coord) {
    farr x = as_n3(coord, "coord");
    const float* p = x.data();
    const int64_t n = x.shape(0);
    py::gil_scoped_release nogil;
    check(hignn_nbl_update_coord(l_, p, n));
  }
  void set_two_body_epsilon(float e) { check(hignn_nbl_set_two_body_epsilon(l_, e)); }
  void set_three_body_epsilon(float e) { check(hignn_nbl_set_three_body_epsilon(l_, e)); }
  void build_two_body_info() {
    py::gil_scoped_release nogil;
    check(hignn_nbl_build_two_body_info(l_));
  }
  void build_three_body_info() {
    py::gil_scoped_release nogil;
    check(hignn_nbl_build_three_body_info(l_));
  }
  py::array_t<uint64_t> get(int kind) { return fetch(kind, false, nullptr, 0); }
  py::array_t<uint64_t> get_by_index(int kind, py::array index) {
    using uarr = py::array_t<uint64_t, py::array::c_style | py::array::forcecast>;
    uarr idx = uarr::ensure(index);
    if (!idx || idx.ndim() != 1) throw std::invalid_argument("target index must be a 1-D integer array");
    return fetch(kind, true, idx.data(), idx.shape(0));
  }

 private:
  py::array_t<uint64_t> fetch(int kind, bool by_index, const uint64_t* idx, int64_t m) {
    const py::ssize_t rows = kind == HIGNN_EDGES_THREE_BODY ? 3 : 2;
    int64_t e = 0;
    check(hignn_nbl_get_edge_info(l_, kind, by_index, idx, m, nullptr, 0, &e));
    py::array_t<uint64_t> out({rows, (py::ssize_t)e});
    uint64_t* o = out.mutable_data();
    {
      py::gil_scoped_release nogil;
      check(hignn_nbl_get_edge_info(l_, kind, by_index, idx, m, o, rows * e, &e));
    }
    return out;
  }
  hignn_nbl* l_ = nullptr;
};

}  // namespace

PYBIND11_MODULE(hignn, m) {
  m.doc() = "B200-native H-HIGNN mobility matvec (drop-in for the reference's hignn module)";
  m.def("Init", [] {}, "No-op: the native library initialises itself (the reference starts MPI and Kokkos)");
  m.def("Finalize", [] {}, "No-op counterpart of Init");

  py::class_<HignnModel>(m, "HignnModel")
      .def(py::init<py::array, int>())
      .def("load_two_body_model", &HignnModel::load_two_body_model)
      .def("load_three_body_model", &HignnModel::load_three_body_model)
      .def("set_epsilon", [](HignnModel& s, double v) { s.set(HIGNN_P_EPSILON, v); })
      .def("set_eta", [](HignnModel& s, double v) { s.set(HIGNN_P_ETA, v); })
      .def("set_max_iter", [](HignnModel& s, int v) { s.set(HIGNN_P_MAX_ITER, v); })
      .def("set_mat_pool_size_factor", [](HignnModel& s, int v) { s.set(HIGNN_P_MAT_POOL_SIZE_FACTOR, v); })
      .def("set_max_far_dot_work_node_size",
           [](HignnModel& s, int v) { s.set(HIGNN_P_MAX_FAR_DOT_WORK_NODE_SIZE, v); })
      .def("set_max_relative_coord", [](HignnModel& s, size_t v) { s.set(HIGNN_P_MAX_RELATIVE_COORD, (double)v); })
      .def("set_post_check_flag", [](HignnModel& s, bool v) { s.set(HIGNN_P_POST_CHECK_FLAG, v); })
      .def("set_use_symmetry_flag", [](HignnModel& s, bool v) { s.set(HIGNN_P_USE_SYMMETRY, v); })
      .def("set_max_far_field_distance", [](HignnModel& s, double v) { s.set(HIGNN_P_MAX_FAR_FIELD_DISTANCE, v); })
      .def("set_precision", [](HignnModel& s, int v) { s.set(HIGNN_P_PRECISION, v); })
      .def("set_param", &HignnModel::set)
      .def("get_param", &HignnModel::get)
      .def("update_coord", &HignnModel::update_coord)
      .def("update_coord_keep_tree", &HignnModel::update_coord_keep_tree)
      .def("dot", &HignnModel::dot)
      .def("dense_dot", &HignnModel::dense_dot)
      .def("stats", &HignnModel::stats);

  py::class_<PotentialForce>(m, "PotentialForce")
      .def(py::init())
      .def("set_periodic", &PotentialForce::set_periodic, py::arg("isPeriodicBoundary") = false)
      .def("set_domain", &PotentialForce::set_domain)
      .def("set_two_body_epsilon", &PotentialForce::set_two_body_epsilon)
      .def("set_parameters", &PotentialForce::set_parameters)
      .def("get_potential_force", &PotentialForce::get_potential_force);

  py::class_<NeighborLists>(m, "NeighborLists")
      .def(py::init())
      .def("set_periodic", &NeighborLists::set_periodic, py::arg("isPeriodicBoundary") = false)
      .def("set_domain", &NeighborLists::set_domain)
      .def("update_coord", &NeighborLists::update_coord)
      .def("set_two_body_epsilon", &NeighborLists::set_two_body_epsilon)
      .def("set_three_body_epsilon", &NeighborLists::set_three_body_epsilon)
      .def("get_two_body_edge_info", [](NeighborLists& l) { return l.get(HIGNN_EDGES_TWO_BODY); })
      .def("get_two_body_edge_info_by_index",
           [](NeighborLists& l, py::array i) { return l.get_by_index(HIGNN_EDGES_TWO_BODY, i); })
      .def("get_three_body_edge_info", [](NeighborLists& l) { return l.get(HIGNN_EDGES_THREE_BODY); })
      .def("get_three_body_edge_info_by_index",
           [](NeighborLists& l, py::array i) { return l.get_by_index(HIGNN_EDGES_THREE_BODY, i); })
      .def("get_three_body_edge_self_info", [](NeighborLists& l) { return l.get(HIGNN_EDGES_THREE_BODY_SELF); })
      .def("get_three_body_edge_self_info_by_index",
           [](NeighborLists& l, py::array i) { return l.get_by_index(HIGNN_EDGES_THREE_BODY_SELF, i); })
      .def("build_two_body_info", &NeighborLists::build_two_body_info)
      .def("build_three_body_info", &NeighborLists::build_three_body_info);

  py::class_<ExplicitEuler>(m, "ExplicitEuler")
      .def(py::init())
      .def("set_time_step", &ExplicitEuler::set_time_step)
      .def("set_final_time", &ExplicitEuler::set_final_time)
      .def("set_num_rigid_body", &ExplicitEuler::set_num_rigid_body)
      .def("set_velocity_func", &ExplicitEuler::set_velocity_func)
      .def("set_output_func", &ExplicitEuler::set_output_func)
      .def("set_x_lim", [](ExplicitEuler& s, py::list l) { s.set_lim(0, l); })
      .def("set_y_lim", [](ExplicitEuler& s, py::list l) { s.set_lim(1, l); })
      .def("set_z_lim", [](ExplicitEuler& s, py::list l) { s.set_lim(2, l); })
      .def("set_output_step", &ExplicitEuler::set_output_step)
      .def("initialize", &ExplicitEuler::initialize)
      .def("run", &ExplicitEuler::run)
      .def("get_func_count", &ExplicitEuler::get_func_count);

  py::class_<ExplicitRk4>(m, "ExplicitRk4")
      .def(py::init())
      .def("set_time_step", &ExplicitRk4::set_time_step)
      .def("set_threshold", &ExplicitRk4::set_threshold)
      .def("set_final_time", &ExplicitRk4::set_final_time)
      .def("set_num_rigid_body", &ExplicitRk4::set_num_rigid_body)
      .def("set_velocity_func", &ExplicitRk4::set_velocity_func)
      .def("set_output_func", &ExplicitRk4::set_output_func)
      .def("set_x_lim", [](ExplicitRk4& s, py::list l) { s.set_lim(0, l); })
      .def("set_y_lim", [](ExplicitRk4& s, py::list l) { s.set_lim(1, l); })
      .def("set_z_lim", [](ExplicitRk4& s, py::list l) { s.set_lim(2, l); })
      .def("set_output_step", &ExplicitRk4::set_output_step)
      .def("initialize", &ExplicitRk4::initialize)
      .def("run", &ExplicitRk4::run)
      .def("get_func_count", &ExplicitRk4::get_func_count);
}
