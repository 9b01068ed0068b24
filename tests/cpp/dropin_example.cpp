// A simulation written the way the reference's examples are
// (Examples/src/Wedge.cpp:20-82), with the Tspeed classes swapped for
// tspeed_gpu. Used by tests/test_gpu_cpp_dropin.py.
//
// usage: dropin_example mesh.msh rcv.txt outprefix N penalty dt nsteps sx sy f0 t0 amp dir
//                       nreg [region lambda mu rho]... [ba]
// A trailing "ba" selects the BoundaryAdapted space (Examples/src/Lamb.cpp:26).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "tspeed_gpu.hpp"

using namespace tspeed_gpu;

int main(int argc, char** argv) {
  if (argc < 15) {
    std::fprintf(stderr, "bad arguments\n");
    return 2;
  }
  int a = 1;
  const std::string mesh = argv[a++], rcv = argv[a++], out = argv[a++];
  const int N = std::atoi(argv[a++]);
  const double pen = std::atof(argv[a++]), dt = std::atof(argv[a++]);
  const int nsteps = std::atoi(argv[a++]);
  const double sx = std::atof(argv[a++]), sy = std::atof(argv[a++]);
  const double f0 = std::atof(argv[a++]), t0 = std::atof(argv[a++]), amp = std::atof(argv[a++]);
  const int dir = std::atoi(argv[a++]);
  const int nreg = std::atoi(argv[a++]);
  try {
    Mesh_ptr Th(new Mesh(mesh));
    const int nreg_args = 4 * nreg;
    const bool ba = argc > a + nreg_args && std::string(argv[a + nreg_args]) == "ba";
    FESpace_ptr Xh(new FESpace(Th, N, ba ? TSP_BASIS_BOUNDARY_ADAPTED : TSP_BASIS_DUBINER));
    Parameters p(Th);
    for (int r = 0; r < nreg; ++r) {
      const unsigned id = unsigned(std::atoi(argv[a++]));
      p.setp("lambda", id, std::atof(argv[a++]));
      p.setp("mu", id, std::atof(argv[a++]));
      p.setp("rho", id, std::atof(argv[a++]));
    }
    Receivers r2(Xh, rcv);
    Force_ptr f(new PointWiseForce(
        [=](const double& t) {
          const double v = amp * ((1 - 2 * M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)) *
                                  std::exp(-M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)));
          return std::array<double, 2>{{dir == 0 ? v : 0.0, dir == 1 ? v : 0.0}};
        },
        Point(sx, sy), Xh));
    LeapFrog TA(Xh, p, r2);
    TA.set_dt(dt);
    TA.set_tmax((nsteps + 0.5) * dt);
    TA.add_force(f);
    TA.set_penalty(pen);
    TA.set_initial_u(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
    TA.set_initial_v(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
    TA.first_step();
    TA.eval_receivers();
    int steps = 1;
    while (TA.is_running()) {
      TA.step();
      TA.eval_receivers();
      ++steps;
    }
    TA.write_receivers(out);
    const std::vector<double>& u = TA.u();
    double s = 0;
    for (double v : u) s += v * v;
    std::printf("steps %d norm %.17g\n", steps, std::sqrt(s));
    // FESpace outputs (FESpace_imp.hpp:70-133): on the host from u, and from
    // the device state.
    auto zero = [](double, double) { return std::array<double, 2>{{0.0, 0.0}}; };
    Xh->points_out(out + ".points");
    Xh->field_out(out + ".host.", u, unsigned(steps));
    TA.field_out(out + ".dev.", unsigned(steps));
    std::printf("l2 %.17g %.17g\n", Xh->L2error(zero, u), TA.L2error(zero));
  } catch (const Error& e) {
    std::fprintf(stderr, "tspeed_gpu error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}
