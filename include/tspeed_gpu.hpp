// tspeed_gpu.hpp: C++ face of the tspeed_b200 engine with the surface of the
// reference's time-loop classes (namespace Tspeed in carlomr/tspeed), so that
// a simulation written against the reference switches its stepping to a B200
// by renaming the namespace:
//
//   Mesh_ptr Th(new Mesh("wedge.msh"));            // Mesh.hpp:47
//   FESpace_ptr Xh(new FESpace(Th, 5));            // FESpace<5> (FESpace.hpp:37), degree at run time
//   Parameters p(Th); p.setp("rho", 1, 2000);      // Parameters.cpp:23-36
//   Receivers r(Xh, "wedge.rcv");                  // Receivers_imp.hpp:61-82
//   Force_ptr f(new PointWiseForce(fun, Point(1500, 1950), Xh));   // Force_imp.hpp:23-31
//   LeapFrog TA(Xh, p, r);                         // TimeAdvance_imp.hpp:29-33
//   TA.set_dt(dt); TA.set_tmax(tmax); TA.add_force(f); TA.set_penalty(c);
//   TA.set_initial_u(Xh, u0); TA.set_initial_v(Xh, v0);
//   TA.first_step(); TA.eval_receivers();
//   while (TA.is_running()) { TA.step(); TA.eval_receivers(); }
//   TA.write_receivers("out/wedge");
//
// Header-only; link with -ltspeed_b200 (include/tspeed_b200.h is the ABI).
// Differences from the reference, all deliberate:
//   * set_penalty takes effect (the operator is built at first_step); the
//     reference builds B in the constructor with its default penalty 2
//     (TimeAdvance_imp.hpp:27,32), so its set_penalty calls are no-ops;
//   * errors throw tspeed_gpu::Error instead of calling exit();
//   * write_receivers writes every sample taken by eval_receivers (the
//     reference's Receivers::add resizes its storage non-conservatively,
//     Receivers.cpp:28, and loses earlier samples);
//   * the degree N is a constructor argument instead of a template parameter;
//     only the default Gauss<N+1> rule and Dubiner<N> basis exist.
#ifndef TSPEED_GPU_HPP
#define TSPEED_GPU_HPP 1

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "tspeed_b200.h"

namespace tspeed_gpu {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const tsp_handle* h = nullptr) {
  if (rc != TSP_OK) throw Error(rc, tsp_last_error(h));
}

struct Point {
  Point(double x = 0, double y = 0) : px(x), py(y) {}
  double x() const { return px; }
  double y() const { return py; }
  double px, py;
};

// Mesh (Mesh.hpp:35-112): Gmsh 2.2 triangles, region = elementary tag.
class Mesh {
 public:
  explicit Mesh(const std::string& fileName) : fname_(fileName) {
    int32_t nv = 0, ne = 0;
    check(tsp_gmsh_read(fileName.c_str(), &nv, nullptr, &ne, nullptr, nullptr));
    xy_.resize(size_t(nv) * 2);
    tri_.resize(size_t(ne) * 3);
    region_.resize(ne);
    check(tsp_gmsh_read(fileName.c_str(), &nv, xy_.data(), &ne, tri_.data(), region_.data()));
  }
  Mesh(std::vector<double> xy, std::vector<int32_t> tri, std::vector<int32_t> region)
      : xy_(std::move(xy)), tri_(std::move(tri)), region_(std::move(region)) {}
  unsigned ne() const { return unsigned(tri_.size() / 3); }
  unsigned nverts() const { return unsigned(xy_.size() / 2); }
  const std::vector<double>& xy() const { return xy_; }
  const std::vector<int32_t>& tri() const { return tri_; }
  const std::vector<int32_t>& region() const { return region_; }

 private:
  std::string fname_;
  std::vector<double> xy_;
  std::vector<int32_t> tri_, region_;
};
typedef std::shared_ptr<Mesh> Mesh_ptr;

// FESpace<N, Gauss<N+1>, Dubiner<N>> (FESpace.hpp:37-180).
// FESpace<N> (Dubiner<N>, the reference default) or, with
// TSP_BASIS_BOUNDARY_ADAPTED, FESpace<N, Dunavant<2N>, BoundaryAdapted<N>>
// (Examples/src/Lamb.cpp:26).
class FESpace {
 public:
  FESpace(Mesh_ptr m, int N, tsp_basis basis = TSP_BASIS_DUBINER) : mesh_(std::move(m)), N_(N), basis_(basis) {
    if (N < 1 || N > 8) throw Error(TSP_ERR_UNSUPPORTED, "degree N must be in 1..8");
  }
  tsp_basis basis() const { return basis_; }
  Mesh_ptr mesh() const { return mesh_; }
  int degree() const { return N_; }
  unsigned nln() const { return unsigned((N_ + 1) * (N_ + 2) / 2); }
  unsigned ne() const { return mesh_->ne(); }
  // FESpace::transform (FESpace_imp.hpp:136-179), reference layout.
  std::vector<double> transform(const std::function<std::array<double, 2>(double, double)>& fun) const {
    const int32_t ne = int32_t(mesh_->ne()), nq = (N_ + 1) * (N_ + 1);
    std::vector<double> pts(size_t(ne) * nq * 2), vals(size_t(ne) * nq * 2), out(2 * size_t(ne) * nln());
    check(tsp_quadrature_points(N_, int32_t(mesh_->nverts()), mesh_->xy().data(), ne, mesh_->tri().data(),
                                pts.data()));
    for (size_t q = 0; q < size_t(ne) * nq; ++q) {
      const std::array<double, 2> f = fun(pts[2 * q], pts[2 * q + 1]);
      vals[2 * q] = f[0];
      vals[2 * q + 1] = f[1];
    }
    check(tsp_project_basis(N_, basis_, int32_t(mesh_->nverts()), mesh_->xy().data(), ne, mesh_->tri().data(),
                            vals.data(), out.data()));
    return out;
  }
  // FESpace::points_out (FESpace_imp.hpp:70-84).
  void points_out(const std::string& fname) const {
    check(tsp_points_out(int32_t(mesh_->nverts()), mesh_->xy().data(), int32_t(mesh_->ne()), mesh_->tri().data(),
                         fname.c_str()));
  }
  // FESpace::field_out (FESpace_imp.hpp:85-105) of a host vector uh
  // (reference layout); LeapFrog::field_out evaluates the device state.
  void field_out(const std::string& fname, const std::vector<double>& uh, unsigned step) const {
    static const double pts[8] = {0.2, 0.2, 0.8, 0.2, 0.2, 0.8, 0.5, 0.5};
    const size_t Np = nln(), ne = mesh_->ne();
    std::vector<double> V(4 * Np);
    check(tsp_eval_basis(N_, basis_, 4, pts, V.data()));
    std::ofstream o(fname + "u_" + std::to_string(step) + ".field");
    for (size_t e = 0; e < ne; ++e)
      for (int q = 0; q < 4; ++q) {
        double vx = 0.0, vy = 0.0;
        for (size_t i = 0; i < Np; ++i) {
          vx += V[q * Np + i] * uh[e * Np + i];
          vy += V[q * Np + i] * uh[ne * Np + e * Np + i];
        }
        o << vx << " " << vy << std::endl;
      }
  }
  // FESpace::L2error (FESpace_imp.hpp:107-133) of a host vector uh, on the
  // collapsed Gauss<N+1> rule.
  double L2error(const std::function<std::array<double, 2>(double, double)>& uex,
                 const std::vector<double>& uh) const {
    const int32_t ne = int32_t(mesh_->ne()), nq = (N_ + 1) * (N_ + 1);
    const size_t Np = nln();
    std::vector<double> r(2 * size_t(nq)), w(nq), B(size_t(nq) * Np), pts(size_t(ne) * nq * 2);
    check(tsp_quadrature_rule(N_, r.data(), w.data()));
    check(tsp_eval_basis(N_, basis_, nq, r.data(), B.data()));
    check(tsp_quadrature_points(N_, int32_t(mesh_->nverts()), mesh_->xy().data(), ne, mesh_->tri().data(),
                                pts.data()));
    const std::vector<double> det = detJ();
    double err = 0.0;
    for (int32_t e = 0; e < ne; ++e) {
      double loc = 0.0;
      for (int32_t q = 0; q < nq; ++q) {
        double ax = 0.0, ay = 0.0;
        for (size_t i = 0; i < Np; ++i) {
          ax += B[q * Np + i] * uh[size_t(e) * Np + i];
          ay += B[q * Np + i] * uh[size_t(ne) * Np + size_t(e) * Np + i];
        }
        const size_t k = size_t(e) * nq + q;
        const std::array<double, 2> f = uex(pts[2 * k], pts[2 * k + 1]);
        loc += ((ax - f[0]) * (ax - f[0]) + (ay - f[1]) * (ay - f[1])) * w[q];
      }
      err += loc * det[e];
    }
    return std::sqrt(err);
  }
  // Signed Jacobian determinants (Geometry.cpp:188-192).
  std::vector<double> detJ() const {
    const size_t ne = mesh_->ne();
    std::vector<double> d(ne);
    const std::vector<double>& xy = mesh_->xy();
    const std::vector<int32_t>& t = mesh_->tri();
    for (size_t e = 0; e < ne; ++e) {
      const double* p0 = &xy[2 * size_t(t[3 * e])];
      const double* p1 = &xy[2 * size_t(t[3 * e + 1])];
      const double* p2 = &xy[2 * size_t(t[3 * e + 2])];
      d[e] = (p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]);
    }
    return d;
  }

 private:
  Mesh_ptr mesh_;
  int N_;
  tsp_basis basis_;
};
typedef std::shared_ptr<FESpace> FESpace_ptr;

// Parameters (FESpace.hpp:194-247): per-element lambda, mu, rho set by region.
class Parameters {
 public:
  explicit Parameters(Mesh_ptr m)
      : mesh_(std::move(m)), v_{{"lambda", std::vector<double>(mesh_->ne(), 0.0)},
                                {"mu", std::vector<double>(mesh_->ne(), 0.0)},
                                {"rho", std::vector<double>(mesh_->ne(), 0.0)}} {}
  void setp(const std::string& p, unsigned lab, double value) {
    auto it = v_.find(p);
    if (it == v_.end()) throw Error(TSP_ERR_ARG, "unknown parameter " + p);
    for (unsigned e = 0; e < mesh_->ne(); ++e)
      if (unsigned(mesh_->region()[e]) == lab) it->second[e] = value;
  }
  // Per-element setter (the reference only offers per-region setp).
  void set_element(unsigned e, double lambda, double mu, double rho) {
    v_["lambda"][e] = lambda;
    v_["mu"][e] = mu;
    v_["rho"][e] = rho;
  }
  double lambda(int i) const { return v_.at("lambda")[i]; }
  double mu(int i) const { return v_.at("mu")[i]; }
  double rho(int i) const { return v_.at("rho")[i]; }
  const std::vector<double>& all(const std::string& p) const { return v_.at(p); }

 private:
  Mesh_ptr mesh_;
  std::map<std::string, std::vector<double>> v_;
};

// Receivers (Receivers.hpp:77-121): "x y" lines; located at construction of
// the LeapFrog (first element containing the point, Receivers_imp.hpp:34-51).
class Receivers {
 public:
  Receivers(FESpace_ptr, const std::string& fname) {
    std::ifstream f(fname);
    if (!f.is_open()) throw Error(TSP_ERR_ARG, "Unable to open file " + fname);
    double x, y;
    while (f >> x >> y) pts_.push_back({x, y});
  }
  Receivers(FESpace_ptr, const Point& p) { pts_.push_back({p.x(), p.y()}); }
  unsigned size() const { return unsigned(pts_.size()); }
  const std::vector<std::array<double, 2>>& points() const { return pts_; }

 private:
  std::vector<std::array<double, 2>> pts_;
};

// Force / PointWiseForce (Force.hpp:33-86).
class Force {
 public:
  virtual ~Force() {}
  virtual std::array<double, 2> value(double t) const = 0;
  virtual Point point() const = 0;
};
typedef std::shared_ptr<Force> Force_ptr;

class PointWiseForce : public Force {
 public:
  PointWiseForce(std::function<std::array<double, 2>(const double&)> f, Point p, FESpace_ptr)
      : f_(std::move(f)), p_(p) {}
  std::array<double, 2> value(double t) const override { return f_(t); }
  Point point() const override { return p_; }

 private:
  std::function<std::array<double, 2>(const double&)> f_;
  Point p_;
};

// LeapFrog (TimeAdvance.hpp:123-256) on the GPU.
class LeapFrog {
 public:
  LeapFrog(FESpace_ptr Xh, const Parameters& p, const Receivers& r, int precision = TSP_PREC_FP64, int device = 0)
      : Xh_(std::move(Xh)), lam_(p.all("lambda")), mu_(p.all("mu")), rho_(p.all("rho")), rcv_(r),
        precision_(precision), device_(device) {}
  ~LeapFrog() { tsp_destroy(h_); }
  LeapFrog(const LeapFrog&) = delete;
  LeapFrog& operator=(const LeapFrog&) = delete;

  void set_dt(double dt) { dt_ = dt; }
  void set_tmax(double tmax) { tmax_ = tmax; }
  void set_penalty(double p) { penalty_ = p; }
  void add_force(Force_ptr f) { force_ = std::move(f); }
  void set_initial_u(FESpace_ptr Xh, std::function<std::array<double, 2>(double, double)> fun) {
    u0_ = Xh->transform(fun);
  }
  void set_initial_v(FESpace_ptr Xh, std::function<std::array<double, 2>(double, double)> fun) {
    v0_ = Xh->transform(fun);
  }

  // LeapFrog::first_step (TimeAdvance.cpp:24-39). Builds the operator.
  void first_step() {
    build();
    check(tsp_set_initial(h_, 0, u0_.empty() ? nullptr : u0_.data(), v0_.empty() ? nullptr : v0_.data()), h_);
    check(tsp_first_step(h_), h_);
    last_time_ = dt_;
    steps_ = 1;
    pending_ = 0;
    completed_ = false;
    dirty_ = true;
  }
  // LeapFrog::step (TimeAdvance.cpp:41-59). The step is queued: steps run on
  // the device as one graph-replayed tsp_run when something reads the state
  // (u(), field_out, L2error, write_receivers, handle()), so a loop of
  // step() calls costs what tsp_run does. The time and is_running() follow
  // the reference's accumulation at once (TimeAdvance.cpp:46, 56-57).
  void step() {
    if (!h_) throw Error(TSP_ERR_STATE, "step before first_step");
    ++pending_;
    ++steps_;
    const double t = last_time_ + dt_;
    last_time_ = t;
    if (t >= tmax_ - dt_) completed_ = true;  // TimeAdvance.cpp:56-57
    dirty_ = true;
  }
  bool is_running() const { return !completed_; }
  double last_time() const { return last_time_; }
  // Runs the queued steps (errors of queued steps surface here).
  void flush() {
    if (pending_ > 0) {
      const int64_t n = pending_;
      pending_ = 0;
      check(tsp_run(h_, n), h_);
    }
  }
  const std::vector<double>& u() {
    flush();
    if (dirty_) {
      uh_.resize(2 * size_t(Xh_->ne()) * Xh_->nln());
      check(tsp_get_u(h_, 0, uh_.data()), h_);
      dirty_ = false;
    }
    return uh_;
  }
  const std::vector<double>& get_uh() { return u(); }
  // Xh->field_out(fname, u(), step) and Xh->L2error(uex, u()) evaluated on
  // the device state.
  void field_out(const std::string& fname, unsigned step) {
    flush();
    check(tsp_write_field(h_, 0, fname.c_str(), step), h_);
  }
  double L2error(const std::function<std::array<double, 2>(double, double)>& uex) {
    flush();
    const Mesh& m = *Xh_->mesh();
    const int32_t ne = int32_t(m.ne()), nq = (Xh_->degree() + 1) * (Xh_->degree() + 1);
    std::vector<double> pts(size_t(ne) * nq * 2), ex(size_t(ne) * nq * 2);
    check(tsp_quadrature_points(Xh_->degree(), int32_t(m.nverts()), m.xy().data(), ne, m.tri().data(), pts.data()));
    for (size_t k = 0; k < size_t(ne) * nq; ++k) {
      const std::array<double, 2> f = uex(pts[2 * k], pts[2 * k + 1]);
      ex[2 * k] = f[0];
      ex[2 * k + 1] = f[1];
    }
    double err = 0.0;
    check(tsp_l2_error(h_, 0, ex.data(), &err), h_);
    return err;
  }
  // TimeAdvance::eval_receivers (TimeAdvance.cpp:68-79): the device samples
  // every step; this records which steps are written out (no device work).
  void eval_receivers() {
    if (!h_) throw Error(TSP_ERR_STATE, "eval_receivers before first_step");
    sampled_.push_back(steps_ - 1);
  }
  // Receivers::write (Receivers.cpp:32-46): <fn>_rcv_<i>.out, "ux uy" lines.
  // The samples of every recorded step come back in one read.
  void write_receivers(const std::string& fn) {
    flush();
    const unsigned nr = rcv_.size();
    std::vector<std::vector<std::array<double, 2>>> rows(nr);
    int64_t nk = 0;
    for (int64_t k : sampled_) nk = std::max<int64_t>(nk, k + 1);
    if (nr > 0 && nk > 0) {
      if (nk > seis_cap_) throw Error(TSP_ERR_STATE, "receiver samples beyond the recorded run length");
      std::vector<double> buf(size_t(nk) * nr * 2);
      check(tsp_get_seismograms(h_, 0, nk, buf.data()), h_);
      for (int64_t k : sampled_)
        for (unsigned i = 0; i < nr; ++i) rows[i].push_back({buf[(size_t(k) * nr + i) * 2], buf[(size_t(k) * nr + i) * 2 + 1]});
    }
    for (unsigned i = 0; i < nr; ++i) {
      std::ofstream o(fn + "_rcv_" + std::to_string(i) + ".out");
      if (!o.is_open()) throw Error(TSP_ERR_ARG, "File " + fn + "_rcv_" + std::to_string(i) + ".out may not be opened");
      o.precision(17);
      for (auto& v : rows[i]) o << v[0] << " " << v[1] << "\n";
    }
  }
  // The engine handle, with every queued step run.
  tsp_handle* handle() {
    flush();
    return h_;
  }

 private:
  void build() {
    if (h_) throw Error(TSP_ERR_STATE, "first_step called twice");
    if (!(dt_ > 0)) throw Error(TSP_ERR_STATE, "set_dt before first_step");
    if (!force_) throw Error(TSP_ERR_STATE, "add_force before first_step");
    const Mesh& m = *Xh_->mesh();
    const Point sp = force_->point();
    const double sxy[2] = {sp.x(), sp.y()};
    std::vector<double> rxy;
    for (auto& q : rcv_.points()) {
      rxy.push_back(q[0]);
      rxy.push_back(q[1]);
    }
    tsp_problem P = {};
    P.nverts = int32_t(m.nverts());
    P.xy = m.xy().data();
    P.ne = int32_t(m.ne());
    P.tri = m.tri().data();
    P.N = Xh_->degree();
    P.lambda = lam_.data();
    P.mu = mu_.data();
    P.rho = rho_.data();
    P.penalty = penalty_;
    P.precision = precision_;
    P.op_kind = TSP_OP_EXPLICIT;
    P.nshots = 1;
    P.src_xy = sxy;
    P.nrcv = int32_t(rcv_.size());
    P.rcv_xy = rxy.empty() ? nullptr : rxy.data();
    P.device = device_;
    P.basis = Xh_->basis();
    check(tsp_create(&P, &h_));
    check(tsp_set_dt(h_, dt_), h_);
    // Force table over the run (time accumulation of TimeAdvance.cpp:46).
    const int64_t n = tmax_ > 0 ? int64_t(std::ceil(tmax_ / dt_)) + 2 : 1;
    std::vector<double> t(n), F(2 * size_t(n));
    check(tsp_force_times(dt_, n, t.data()));
    for (int64_t k = 0; k < n; ++k) {
      const std::array<double, 2> v = force_->value(t[k]);
      F[2 * k] = v[0];
      F[2 * k + 1] = v[1];
    }
    check(tsp_set_force_table(h_, 0, F.data(), n), h_);
    check(tsp_set_seismogram_capacity(h_, n), h_);
    seis_cap_ = n;
  }

  FESpace_ptr Xh_;
  std::vector<double> lam_, mu_, rho_;
  Receivers rcv_;
  int precision_, device_;
  tsp_handle* h_ = nullptr;
  double dt_ = 0, tmax_ = 0, penalty_ = 2.0, last_time_ = 0;
  int64_t steps_ = 0, pending_ = 0, seis_cap_ = 0;
  bool completed_ = false, dirty_ = true;
  Force_ptr force_;
  std::vector<double> u0_, v0_, uh_;
  std::vector<int64_t> sampled_;
};

}  // namespace tspeed_gpu

#endif
