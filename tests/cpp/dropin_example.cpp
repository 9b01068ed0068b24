// A simulation written the way the reference's examples are
// (Examples/src/Wedge.cpp:20-82), with the Tspeed classes swapped for
// tspeed_gpu. Used by tests/test_gpu_cpp_dropin.py.
//
// usage: dropin_example mesh.msh rcv.txt outprefix N penalty dt nsteps sx sy f0 t0 amp dir
//                       nreg [region lambda mu rho]... [ba] [timing]
// A trailing "ba" selects the BoundaryAdapted space (Examples/src/Lamb.cpp:26).
// A trailing "timing" also times the stepping loop (step() and
// eval_receivers() calls, then write_receivers) against the same run done
// with one tsp_run call on the engine handle, both wall-clock.
#include <chrono>
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
    bool ba = false, timing = false;
    for (int i = a + nreg_args; i < argc; ++i) {
      ba = ba || std::string(argv[i]) == "ba";
      timing = timing || std::string(argv[i]) == "timing";
    }
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
    auto setup = [&](LeapFrog& T) {
      T.set_dt(dt);
      T.set_tmax((nsteps + 0.5) * dt);
      T.add_force(f);
      T.set_penalty(pen);
      T.set_initial_u(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
      T.set_initial_v(Xh, [](double, double) { return std::array<double, 2>{{0, 0}}; });
    };
    typedef std::chrono::steady_clock clk;
    LeapFrog TA(Xh, p, r2);
    setup(TA);
    TA.first_step();
    const auto t0 = clk::now();
    TA.eval_receivers();
    int steps = 1;
    while (TA.is_running()) {
      TA.step();
      TA.eval_receivers();
      ++steps;
    }
    TA.write_receivers(out);
    const double loop_s = std::chrono::duration<double>(clk::now() - t0).count();
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
    if (timing) {
      // The same run on a second handle with one tsp_run call and one
      // read-back of every receiver sample; both runs once more to time
      // them warm (graphs instantiated, allocator pool filled).
      double best_run = 1e30, best_loop = loop_s;
      for (int rep = 0; rep < 3; ++rep) {
        LeapFrog TB(Xh, p, r2);
        setup(TB);
        TB.first_step();
        tsp_handle* hb = TB.handle();
        const auto t1 = clk::now();
        check(tsp_run(hb, steps - 1), hb);
        std::vector<double> all(size_t(steps) * r2.size() * 2);
        check(tsp_get_seismograms(hb, 0, steps, all.data()), hb);
        best_run = std::min(best_run, std::chrono::duration<double>(clk::now() - t1).count());
        LeapFrog TC(Xh, p, r2);
        setup(TC);
        TC.first_step();
        const auto t2 = clk::now();
        TC.eval_receivers();
        while (TC.is_running()) {
          TC.step();
          TC.eval_receivers();
        }
        TC.write_receivers(out + ".timing");
        best_loop = std::min(best_loop, std::chrono::duration<double>(clk::now() - t2).count());
      }
      std::printf("timing dropin_loop_s %.6f tsp_run_s %.6f\n", best_loop, best_run);
    }
  } catch (const Error& e) {
    std::fprintf(stderr, "tspeed_gpu error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}
