// Reference-oracle harness (test infrastructure; never part of the product).
//
// Compiled together with the reference's own, unmodified lib/src/*.cpp and
// lib/include/*.hpp against the project's Eigen-subset shim
// (oracle/eigen_shim). It runs the reference's public API exactly as
// Examples/src/Wedge.cpp:20-82 does (Mesh -> FESpace<N> -> Parameters ->
// Receivers -> PointWiseForce -> LeapFrog) and dumps golden data:
//   * the operator B blocks (TimeAdvance_imp.hpp:32) in a merged 2Np x 2Np
//     per (row, col) layout, with the block-CSR pattern of MyMat
//     (MyMat.cpp:128-154),
//   * the inverse-mass scalars (Matrices_imp.hpp:187,189) and the reference
//     element's inverse mass matrix (FESpace_imp.hpp:48-68; the identity for
//     the orthonormal Dubiner basis, dense for BoundaryAdapted),
//   * the mesh neighbour tables (Mesh.cpp:33-128),
//   * source / receiver location (Receivers_imp.hpp:34-51),
//   * displacement snapshots and receiver samples of the leap-frog loop
//     (TimeAdvance.cpp:24-59),
//   * the FESpace services around the loop: transform of a fixed field
//     (FESpace_imp.hpp:136-179), L2error (FESpace_imp.hpp:107-133) of that
//     projection and of the final displacement, and the text outputs
//     field_out / points_out (FESpace_imp.hpp:70-106) of the final step.
//
// LeapFrogP re-forms B with the requested penalty. In the reference, B is built
// in the LeapFrog constructor with the default M_penalty(2)
// (TimeAdvance_imp.hpp:27,32), so set_penalty() called afterwards has no
// effect; M_penalty, M_mat and B are protected (TimeAdvance.hpp:214-228).
//
// --basis ba runs the reference with FESpace<N, Dunavant<2N>,
// BoundaryAdapted<N>>, the space of Examples/src/Lamb.cpp:26; the default is
// FESpace<N> = FESpace<N, Gauss<N+1>, Dubiner<N>> (Examples/src/Wedge.cpp).
//
// Receiver samples are taken here, with the same arithmetic as
// TimeAdvance::eval_receivers (TimeAdvance.cpp:68-79): Receivers::add
// resizes its storage non-conservatively every step (Receivers.cpp:28), so
// the reference's own recording cannot be read back.
#include "TSPEED.hpp"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

using namespace Tspeed;

namespace {

struct Args {
  std::string mesh, mat, rcv, out;
  int N = 4;
  double penalty = 2.0;
  double dt = 1e-3;
  long nsteps = 10;
  double tmax = -1;  // if > 0: run the reference's own is_running() loop
  double sx = 0, sy = 0;
  double f0 = 10, t0 = 0.1, amp = 1.0;
  int sdir = 1;
  bool dump_blocks = false;
  bool quiet = true;
  long u_every = 0;  // snapshot interval (0: only first and last)
  bool region_mat = false;
  bool boundary_adapted = false;
  double reg_vals[16][3];
  int reg_ids[16];
  int nreg = 0;
};

void die(const char* m) {
  std::fprintf(stderr, "tsp_ref_run: %s\n", m);
  std::exit(2);
}

template <typename T>
void wr(std::FILE* f, const T* p, size_t n) {
  if (std::fwrite(p, sizeof(T), n, f) != n) die("write failed");
}

// Ricker wavelet in the form of Examples/src/Lamb.cpp:37, scaled by amp.
double ricker(double t, double f0, double t0, double amp) {
  return amp * ((1 - 2 * M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)) *
                exp(-M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)));
}

class LeapFrogP : public LeapFrog {
 public:
  template <int N, typename Q, typename S>
  LeapFrogP(FESpace_ptr<N, Q, S> Xh, Parameters const& p, Receivers const& r, double penalty)
      : LeapFrog(Xh, p, r) {
    M_penalty = penalty;
    B = std::move(M_penalty * N * N * M_mat.getS() + M_mat.getI() + M_mat.getA());
  }
  MyMatMultiDim<MyMat> const& op() const { return B; }
  Matrices& mats() { return M_mat; }
  unsigned int last_step() const { return M_last_step; }
  double last_time() const { return M_last_time; }
};

template <int N, typename Q, typename S>
int run_space(const Args& a) {
  using clk = std::chrono::steady_clock;
  auto t_setup0 = clk::now();
  Mesh_ptr Th(new Mesh(a.mesh));
  const unsigned ne = Th->ne();
  FESpace_ptr<N, Q, S> Xh(new FESpace<N, Q, S>(Th));
  const unsigned nln = Xh->nln();
  Parameters p(Th);
  if (a.region_mat) {
    for (int r = 0; r < a.nreg; ++r) {
      p.setp("lambda", a.reg_ids[r], a.reg_vals[r][0]);
      p.setp("mu", a.reg_ids[r], a.reg_vals[r][1]);
      p.setp("rho", a.reg_ids[r], a.reg_vals[r][2]);
    }
  } else {
    // Per-element materials: the reference only offers per-region setp
    // (Parameters.cpp:23-36); lambda()/mu()/rho() return references into its
    // arrays, which the harness fills directly.
    std::vector<double> m(size_t(ne) * 3);
    std::FILE* f = std::fopen(a.mat.c_str(), "rb");
    if (!f) die("cannot open material file");
    if (std::fread(m.data(), sizeof(double), m.size(), f) != m.size()) die("short material file");
    std::fclose(f);
    for (unsigned e = 0; e < ne; ++e) {
      const_cast<double&>(p.lambda(e)) = m[3 * e + 0];
      const_cast<double&>(p.mu(e)) = m[3 * e + 1];
      const_cast<double&>(p.rho(e)) = m[3 * e + 2];
    }
  }
  Receivers rc(Xh, a.rcv);
  const double f0 = a.f0, t0 = a.t0, amp = a.amp;
  const int sdir = a.sdir;
  std::shared_ptr<PointWiseForce> force(new PointWiseForce(
      [=](const double& t) {
        double v = ricker(t, f0, t0, amp);
        return std::array<double, 2>{{sdir == 0 ? v : 0.0, sdir == 1 ? v : 0.0}};
      },
      Geo::Point(a.sx, a.sy), Xh));
  LeapFrogP TA(Xh, p, rc, a.penalty);
  TA.set_dt(a.dt);
  TA.set_tmax(a.tmax > 0 ? a.tmax : 1e300);
  TA.add_force(force);
  TA.set_initial_u(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
  TA.set_initial_v(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
  double setup_s = std::chrono::duration<double>(clk::now() - t_setup0).count();

  // ---- static dumps ----
  {
    std::FILE* f = std::fopen((a.out + ".mesh.bin").c_str(), "wb");
    if (!f) die("cannot open output");
    int32_t hdr[2] = {int32_t(ne), int32_t(nln)};
    wr(f, hdr, 2);
    for (unsigned e = 0; e < ne; ++e) {
      const Geo::Triangle& t = (*Th)[e];
      int32_t nb[6] = {t.neigh(0), t.neigh(1), t.neigh(2), t.neighedges(0), t.neighedges(1), t.neighedges(2)};
      wr(f, nb, 6);
    }
    for (unsigned e = 0; e < ne; ++e) {
      const Geo::Triangle& t = (*Th)[e];
      double g[5] = {t.detJ(), t.invJac()(0, 0), t.invJac()(1, 0), t.invJac()(0, 1), t.invJac()(1, 1)};
      wr(f, g, 5);
    }
    // Inverse mass: invM blocks are M_ref^-1/(rho*detJ) (Matrices_imp.hpp:187);
    // the scalar 1/(rho*detJ) is their (0,0) entry over M_ref^-1(0,0).
    auto const& invM = TA.mats().getinvM();
    const Eigen::MatrixXd minv_ref = Xh->base_invmass();
    for (unsigned e = 0; e < ne; ++e) {
      double v = invM.component(0).elem(e)(0, 0) / minv_ref(0, 0);
      wr(f, &v, 1);
    }
    // Source location and tabulated basis (PointWiseForce via M_add).
    int32_t se = int32_t(force->elem(0));
    wr(f, &se, 1);
    for (unsigned s = 0; s < nln; ++s) {
      double v = force->shape(0)[s];
      wr(f, &v, 1);
    }
    int32_t nr = int32_t(rc.size());
    wr(f, &nr, 1);
    for (int r = 0; r < nr; ++r) {
      int32_t re = int32_t(rc.elem(r));
      wr(f, &re, 1);
      for (unsigned s = 0; s < nln; ++s) {
        double v = rc.shape(r)[s];
        wr(f, &v, 1);
      }
    }
    for (unsigned i = 0; i < nln; ++i)
      for (unsigned j = 0; j < nln; ++j) {
        double v = minv_ref(i, j);
        wr(f, &v, 1);
      }
    std::fclose(f);
  }
  if (a.dump_blocks) {
    auto const& Bm = TA.op();
    const BaseMat& c00 = Bm.component(0, 0);
    const unsigned nnzb = c00.size();
    std::FILE* f = std::fopen((a.out + ".blocks.bin").c_str(), "wb");
    if (!f) die("cannot open output");
    int32_t hdr[3] = {int32_t(ne), int32_t(nln), int32_t(nnzb)};
    wr(f, hdr, 3);
    std::vector<int32_t> rp(c00.rowInd().begin(), c00.rowInd().end());
    std::vector<int32_t> cp(c00.colInd().begin(), c00.colInd().end());
    wr(f, rp.data(), rp.size());
    wr(f, cp.data(), cp.size());
    const unsigned R = 2 * nln;
    std::vector<double> blk(size_t(R) * R);
    for (unsigned b = 0; b < nnzb; ++b) {
      for (int m = 0; m < 2; ++m)
        for (int n = 0; n < 2; ++n) {
          const Eigen::MatrixXd& M = Bm.component(m, n).elem(b);
          for (unsigned i = 0; i < nln; ++i)
            for (unsigned j = 0; j < nln; ++j) blk[size_t(m * nln + i) * R + n * nln + j] = M(i, j);
        }
      wr(f, blk.data(), blk.size());
    }
    std::fclose(f);
  }

  // ---- time loop ----
  std::FILE* fu = std::fopen((a.out + ".u.bin").c_str(), "wb");
  std::FILE* fs = std::fopen((a.out + ".seis.bin").c_str(), "wb");
  if (!fu || !fs) die("cannot open output");
  auto snap = [&](long step) {
    const Eigen::VectorXd& u = TA.u();
    int64_t s = step;
    wr(fu, &s, 1);
    wr(fu, u.data(), size_t(u.size()));
  };
  auto sample = [&]() {
    const Eigen::VectorXd& u = TA.u();
    for (unsigned i = 0; i < rc.size(); ++i) {
      double xy[2];
      xy[0] = rc.shape(i).matrix().dot(u.segment(rc.elem(i) * nln, nln));
      xy[1] = rc.shape(i).matrix().dot(u.segment(rc.elem(i) * nln + nln * ne, nln));
      wr(fs, xy, 2);
    }
  };
  auto t_loop0 = clk::now();
  TA.first_step();
  sample();
  snap(1);
  long steps = 1;
  if (a.tmax > 0) {
    while (TA.is_running()) {
      TA.step();
      ++steps;
      sample();
      if (a.u_every > 0 && steps % a.u_every == 0) snap(steps);
    }
  } else {
    for (long k = 1; k < a.nsteps; ++k) {
      TA.step();
      ++steps;
      sample();
      if (a.u_every > 0 && steps % a.u_every == 0) snap(steps);
    }
  }
  double loop_s = std::chrono::duration<double>(clk::now() - t_loop0).count();
  if (!(a.u_every > 0 && steps % a.u_every == 0)) snap(steps);
  std::fclose(fu);
  std::fclose(fs);

  // ---- FESpace services ----
  // The projected field: smooth for the Dubiner space (transform and L2error
  // integrate with Gauss<N+1> there); linear for BoundaryAdapted, whose
  // Dunavant<2N> rule then integrates every product exactly as well.
  const bool ba = !S::is_orthonormal;
  auto field = [ba](double x, double y) {
    if (ba) return std::array<double, 2>{{1e-3 + 2e-6 * x - 3e-6 * y, -2e-3 + 1e-6 * x + 4e-6 * y}};
    return std::array<double, 2>{{std::sin(x / 97.0) * std::cos(y / 61.0), 1e-6 * x * y}};
  };
  const Eigen::VectorXd proj = Xh->transform(field);
  {
    std::FILE* f = std::fopen((a.out + ".proj.bin").c_str(), "wb");
    if (!f) die("cannot open output");
    wr(f, proj.data(), size_t(proj.size()));
    std::fclose(f);
  }
  const double l2_proj = Xh->L2error(field, proj);
  const double l2_u = Xh->L2error([](double, double) { return std::array<double, 2>{{0.0, 0.0}}; }, TA.u());
  Xh->field_out(a.out + ".", TA.u(), unsigned(steps));
  Xh->points_out(a.out + ".points");
  std::printf("{\"ne\": %u, \"Np\": %u, \"steps\": %ld, \"last_time\": %.17g, \"setup_s\": %.6f, \"loop_s\": %.6f, "
              "\"l2_proj\": %.17g, \"l2_u\": %.17g}\n",
              ne, nln, steps, TA.last_time(), setup_s, loop_s, l2_proj, l2_u);
  return 0;
}

template <int N>
int run(const Args& a) {
  if (a.boundary_adapted) return run_space<N, Dunavant<2 * N>, BoundaryAdapted<N>>(a);
  return run_space<N, Gauss<N + 1>, Dubiner<N>>(a);
}

}  // namespace

int main(int argc, char** argv) {
  Args a;
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    auto nxt = [&]() -> const char* {
      if (i + 1 >= argc) die("missing value");
      return argv[++i];
    };
    if (k == "--mesh") a.mesh = nxt();
    else if (k == "--mat") a.mat = nxt();
    else if (k == "--rcv") a.rcv = nxt();
    else if (k == "--out") a.out = nxt();
    else if (k == "--N") a.N = std::atoi(nxt());
    else if (k == "--penalty") a.penalty = std::atof(nxt());
    else if (k == "--dt") a.dt = std::atof(nxt());
    else if (k == "--nsteps") a.nsteps = std::atol(nxt());
    else if (k == "--tmax") a.tmax = std::atof(nxt());
    else if (k == "--src") { a.sx = std::atof(nxt()); a.sy = std::atof(nxt()); }
    else if (k == "--ricker") { a.f0 = std::atof(nxt()); a.t0 = std::atof(nxt()); a.amp = std::atof(nxt()); }
    else if (k == "--sdir") a.sdir = std::atoi(nxt());
    else if (k == "--dump-blocks") a.dump_blocks = true;
    else if (k == "--u-every") a.u_every = std::atol(nxt());
    else if (k == "--basis") {
      const std::string b = nxt();
      if (b == "ba") a.boundary_adapted = true;
      else if (b != "dubiner") die("--basis must be dubiner or ba");
    }
    else if (k == "--region") {
      // --region id lambda mu rho (repeatable): per-region setp, as the examples do.
      if (a.nreg >= 16) die("too many regions");
      a.region_mat = true;
      a.reg_ids[a.nreg] = std::atoi(nxt());
      for (int c = 0; c < 3; ++c) a.reg_vals[a.nreg][c] = std::atof(nxt());
      ++a.nreg;
    } else if (k == "--verbose") a.quiet = false;
    else die(("unknown option " + k).c_str());
  }
  if (a.mesh.empty() || a.rcv.empty() || a.out.empty()) die("need --mesh --rcv --out");
  if (!a.region_mat && a.mat.empty()) die("need --mat or --region");
  // The reference prints progress on every step (TimeAdvance.cpp:49); keep it
  // off the JSON result line unless asked for.
  std::streambuf* saved = nullptr;
  std::ofstream devnull;
  if (a.quiet) {
    devnull.open("/dev/null");
    saved = std::cout.rdbuf(devnull.rdbuf());
  }
  std::FILE* real_stdout = stdout;
  (void)real_stdout;
  int rc = 0;
  switch (a.N) {
    case 1: rc = run<1>(a); break;
    case 2: rc = run<2>(a); break;
    case 3: rc = run<3>(a); break;
    case 4: rc = run<4>(a); break;
    case 5: rc = run<5>(a); break;
    case 6: rc = run<6>(a); break;
    case 7: rc = run<7>(a); break;
    case 8: rc = run<8>(a); break;
    default: die("N must be in 1..8");
  }
  if (saved) std::cout.rdbuf(saved);
  return rc;
}
