// Host layer of tspeed_b200 under AddressSanitizer and UndefinedBehaviorSanitizer.
//
// Built by tests/test_host_sanitizers.py with
//   g++ -std=c++17 -fsanitize=address,undefined -fno-sanitize-recover=all
// together with tspeed_b200/csrc/tsp_host.cpp (no CUDA involved) and run on
// the CPU. It drives every host routine the C-ABI uses -- reference tables
// for both bases and N = 1..8, geometry, the O(ne) neighbour search and the
// block-CSR pattern, point location (single and gridded), the Gmsh reader on
// good and malformed files, the volume rule, quadrature points, projection,
// force times and the Ricker wavelet -- and checks invariants of their
// results, so that a sanitizer report or a broken invariant fails the test.
// Usage: host_sanitize <scratch directory>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "tsp_host.h"

namespace {

int g_fail = 0;

void check(bool ok, const char* what) {
  if (!ok) {
    std::fprintf(stderr, "FAILED: %s\n", what);
    ++g_fail;
  }
}

// nx x ny squares over [0,lx] x [0,ly], each split by its diagonal into two
// counter-clockwise triangles; interior vertices jittered by up to 10 % of h.
void jittered_rect(int nx, int ny, double lx, double ly, unsigned seed, std::vector<double>* xy,
                   std::vector<int32_t>* tri) {
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> u(-0.1, 0.1);
  const double hx = lx / nx, hy = ly / ny;
  xy->clear();
  tri->clear();
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      double x = i * hx, y = j * hy;
      if (i > 0 && i < nx && j > 0 && j < ny) {
        x += u(rng) * hx;
        y += u(rng) * hy;
      }
      xy->push_back(x);
      xy->push_back(y);
    }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int32_t a = j * (nx + 1) + i, b = a + 1, c = a + nx + 1, d = c + 1;
      tri->insert(tri->end(), {a, b, d});
      tri->insert(tri->end(), {a, d, c});
    }
}

void write_text(const std::string& path, const std::string& text) {
  std::ofstream f(path);
  f << text;
}

std::string msh_text(const std::vector<double>& xy, const std::vector<int32_t>& tri) {
  std::string s = "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n";
  const size_t nv = xy.size() / 2, ne = tri.size() / 3;
  s += std::to_string(nv) + "\n";
  char buf[128];
  for (size_t v = 0; v < nv; ++v) {
    std::snprintf(buf, sizeof buf, "%zu %.17g %.17g 0\n", v + 1, xy[2 * v], xy[2 * v + 1]);
    s += buf;
  }
  s += "$EndNodes\n$Elements\n" + std::to_string(ne + 1) + "\n";
  s += "1 15 2 0 1 1\n";  // a point element, which the reader skips
  for (size_t e = 0; e < ne; ++e) {
    std::snprintf(buf, sizeof buf, "%zu 2 2 %d %zu %d %d %d\n", e + 2, int(e % 3) + 1, e + 1, tri[3 * e] + 1,
                  tri[3 * e + 1] + 1, tri[3 * e + 2] + 1);
    s += buf;
  }
  s += "$EndElements\n";
  return s;
}

}  // namespace

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";

  // Reference tables: both bases, every degree; the reference mass times its
  // inverse is the identity.
  for (int basis : {tsp::kDubiner, tsp::kBoundaryAdapted})
    for (int N = 1; N <= 8; ++N) {
      const tsp::RefTables t = tsp::make_tables(N, basis);
      const int Np = tsp::np_of(N);
      check(t.Np == Np && t.M.size() == size_t(Np) * Np && t.Minv.size() == t.M.size(), "table sizes");
      double worst = 0.0;
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          double s = 0.0;
          for (int k = 0; k < Np; ++k) s += t.M[i * Np + k] * t.Minv[k * Np + j];
          worst = std::fmax(worst, std::fabs(s - (i == j ? 1.0 : 0.0)));
        }
      check(worst < 1e-9, "reference mass inverse");
      check(t.K.size() == size_t(4) * Np * Np && t.Dx.size() == size_t(18) * Np * Np, "operator table sizes");
    }

  // Geometry, neighbours and the block pattern of a jittered mesh.
  std::vector<double> xy;
  std::vector<int32_t> tri;
  jittered_rect(12, 7, 1200.0, 700.0, 11u, &xy, &tri);
  const int32_t ne = int32_t(tri.size() / 3);
  const tsp::Geometry g = tsp::make_geometry(ne, xy.data(), tri.data());
  for (int32_t e = 0; e < ne; ++e) check(g.detJ[e] > 0.0, "counter-clockwise triangles have positive detJ");
  std::vector<int32_t> neigh(3 * size_t(ne)), nedge(3 * size_t(ne));
  std::string err;
  check(tsp::build_neighbours(ne, tri.data(), neigh.data(), nedge.data(), &err), "neighbour search");
  int interior = 0;
  for (int32_t e = 0; e < ne; ++e)
    for (int l = 0; l < 3; ++l) {
      const int32_t n = neigh[3 * e + l];
      if (n < 0) continue;
      ++interior;
      check(n < ne && neigh[3 * n + nedge[3 * e + l]] == e, "neighbour tables are symmetric");
    }
  std::vector<int32_t> row_ptr, col;
  std::vector<int8_t> bface;
  tsp::bsr_pattern(ne, neigh.data(), &row_ptr, &col, &bface);
  check(int(row_ptr.size()) == ne + 1 && row_ptr[ne] == ne + interior && col.size() == bface.size(),
        "block pattern size nnzb = ne + 2 E_int");
  for (int32_t e = 0; e < ne; ++e) check(col[row_ptr[e]] == e && bface[row_ptr[e]] == -1, "diagonal block first");

  // A clockwise triangle next to its counter-clockwise twin repeats a
  // directed edge: rejected with a message.
  {
    std::vector<int32_t> bad = tri;
    std::swap(bad[1], bad[2]);
    std::string msg;
    std::vector<int32_t> nb(3 * size_t(ne)), ned(3 * size_t(ne));
    check(!tsp::build_neighbours(ne, bad.data(), nb.data(), ned.data(), &msg) && !msg.empty(),
          "a repeated directed edge is rejected");
  }

  // Point location: the gridded search finds the same first-hit element as
  // the element scan, with the same basis values; points outside get -1.
  for (int basis : {tsp::kDubiner, tsp::kBoundaryAdapted}) {
    const int N = 5, Np = tsp::np_of(N);
    std::mt19937 rng(5u);
    std::uniform_real_distribution<double> ux(-50.0, 1250.0), uy(-50.0, 750.0);
    const int npts = 300;
    std::vector<double> pts(2 * npts);
    for (int k = 0; k < npts; ++k) {
      pts[2 * k] = ux(rng);
      pts[2 * k + 1] = uy(rng);
    }
    pts[0] = 0.0;  // a corner vertex and a point on a shared edge
    pts[1] = 0.0;
    pts[2] = 100.0;
    pts[3] = 0.0;
    std::vector<int32_t> elem(npts);
    std::vector<double> phi(size_t(npts) * Np);
    tsp::locate_points(N, ne, xy.data(), tri.data(), g, npts, pts.data(), elem.data(), phi.data(), basis);
    std::vector<double> one(Np);
    for (int k = 0; k < npts; ++k) {
      const int32_t e1 = tsp::locate_point(N, ne, xy.data(), tri.data(), g, pts[2 * k], pts[2 * k + 1], one.data(), basis);
      check(e1 == elem[k], "gridded and scanned point location agree");
      const bool inside = pts[2 * k] >= 0.0 && pts[2 * k] <= 1200.0 && pts[2 * k + 1] >= 0.0 && pts[2 * k + 1] <= 700.0;
      check(inside == (e1 >= 0), "points inside the domain are located, outside ones are not");
      if (e1 >= 0)
        for (int i = 0; i < Np; ++i) check(one[i] == phi[size_t(k) * Np + i], "same basis values");
    }
  }

  // Gmsh 2.2: a written mesh reads back; truncated, unknown-version and
  // out-of-range files are rejected with a message.
  {
    const std::string good = dir + "/ok.msh";
    write_text(good, msh_text(xy, tri));
    std::vector<double> rxy;
    std::vector<int32_t> rtri, region;
    std::string msg;
    check(tsp::gmsh_read(good, &rxy, &rtri, &region, &msg), "Gmsh file reads");
    check(rxy.size() == xy.size() && rtri == tri && int(region.size()) == ne, "Gmsh round trip");
    const std::string text = msh_text(xy, tri);
    const std::string bads[] = {
        text.substr(0, text.size() / 2),                                     // truncated
        "$MeshFormat\n9.9 0 8\n$EndMeshFormat\n",                            // unknown version
        "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n1\n1 0 0 0\n$EndNodes\n"
        "$Elements\n1\n1 2 2 1 1 1 2 7\n$EndElements\n",                     // nodes out of range
        "",                                                                  // empty
    };
    int k = 0;
    for (const std::string& b : bads) {
      const std::string path = dir + "/bad" + std::to_string(k++) + ".msh";
      write_text(path, b);
      std::string m;
      std::vector<double> bx;
      std::vector<int32_t> bt, br;
      check(!tsp::gmsh_read(path, &bx, &bt, &br, &m) && !m.empty(), "malformed Gmsh file rejected");
    }
    std::string m;
    check(!tsp::gmsh_read(dir + "/missing.msh", &rxy, &rtri, &region, &m) && !m.empty(), "missing file rejected");
  }

  // Volume rule, quadrature points and projection: a constant field projects
  // onto the constant mode only (Dubiner), reproducing its value.
  for (int N = 1; N <= 8; ++N) {
    std::vector<double> c, e, w;
    tsp::volume_rule(N, &c, &e, &w);
    double area = 0.0;
    for (double wi : w) area += wi;
    check(std::fabs(area - 0.5) < 1e-12, "volume rule integrates 1 to the reference area");
    const int Q2 = (N + 1) * (N + 1), Np = tsp::np_of(N);
    std::vector<double> qp(size_t(ne) * Q2 * 2), fv(size_t(ne) * Q2 * 2), out(2 * size_t(ne) * Np);
    tsp::quadrature_points(N, ne, xy.data(), tri.data(), qp.data());
    for (size_t q = 0; q < size_t(ne) * Q2; ++q) {
      fv[2 * q] = 2.0;
      fv[2 * q + 1] = -3.0;
      check(qp[2 * q] >= -1e-9 && qp[2 * q] <= 1200.0 + 1e-9, "quadrature points inside the mesh");
    }
    tsp::project(N, ne, xy.data(), tri.data(), fv.data(), out.data());
    std::vector<double> phi(Np);
    tsp::dubiner_phi(N, 1.0 / 3.0, 1.0 / 3.0, phi.data());
    for (int32_t el = 0; el < ne; el += 17) {
      double vx = 0.0, vy = 0.0;
      for (int i = 0; i < Np; ++i) {
        vx += out[size_t(el) * Np + i] * phi[i];
        vy += out[size_t(ne) * Np + size_t(el) * Np + i] * phi[i];
      }
      check(std::fabs(vx - 2.0) < 1e-10 && std::fabs(vy + 3.0) < 1e-10, "constant field projects exactly");
    }
  }

  // Force times: 0 for the first step, then the reference's accumulated
  // last time plus dt (its last time starts at dt after the first step);
  // the Ricker wavelet peaks at t0 with the given amplitude.
  {
    std::vector<double> t(1001);
    tsp::force_times(1e-3, 1001, t.data());
    double acc = 1e-3;
    bool same = t[0] == 0.0;
    for (int k = 1; k < 1001; ++k) {
      acc += 1e-3;
      same = same && t[k] == acc;
    }
    check(same, "force times accumulate dt");
    check(std::fabs(tsp::ricker(0.1, 10.0, 0.1, -2.0) + 2.0) < 1e-15, "Ricker peak");
  }

  if (g_fail) std::fprintf(stderr, "%d check(s) failed\n", g_fail);
  else std::printf("host layer checks passed\n");
  return g_fail ? 1 : 0;
}
