// Host-side setup for the tspeed_b200 engine (see tsp_host.h).
#include "tsp_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <limits>
#include <sstream>
#include <unordered_map>

namespace tsp {

void gauleg(int n, double a, double b, double* x, double* w) {
  // Newton iteration on P_n from the Chebyshev-like initial guess, one root
  // per symmetric pair (QuadratureRule_imp.hpp:23-61).
  const double m = (n + 1.0) / 2.0;
  const double xm = 0.5 * (b + a), xl = 0.5 * (b - a);
  const double eps = std::numeric_limits<double>::epsilon();
  for (int i = 1; i <= m; ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (n + 0.5)), z1, pp;
    do {
      double p1 = 1.0, p2 = 0.0, p3;
      for (int j = 1; j <= n; ++j) {
        p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::abs(z - z1) > eps);
    x[i - 1] = xm - xl * z;
    x[n - i] = xm + xl * z;
    w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp);
    w[n - i] = w[i - 1];
  }
}

double jacobi(int n, int alpha, int beta, double z) {
  if (n < 0) return 0.0;
  if (n == 0) return 1.0;
  const double p1_0 = 0.5 * (alpha - beta + (alpha + beta + 2.0) * z);
  if (n == 1) return p1_0;
  const int apb = alpha + beta;
  double p2 = 1.0, p1 = p1_0, p = p1_0;
  for (int k = 2; k <= n; ++k) {
    const double a1 = 2.0 * k * (k + apb) * (2.0 * k + apb - 2.0);
    const double a2 = (2.0 * k + apb - 1.0) * (alpha * alpha - beta * beta) / a1;
    const double a3 = (2.0 * k + apb - 2.0) * (2.0 * k + apb - 1.0) * (2.0 * k + apb) / a1;
    const double a4 = 2.0 * (k + alpha - 1.0) * (k + beta - 1.0) * (2.0 * k + apb) / a1;
    p = (a2 + a3 * z) * p1 - a4 * p2;
    p2 = p1;
    p1 = p;
  }
  return p;
}

static double cij_of(int i, int j) { return std::sqrt((2.0 * i + 1) * 2.0 * (i + j + 1) / std::pow(4.0, i)); }

void dubiner_phi(int N, double csi, double eta, double* phi) {
  int s = 0;
  const double om = 1 - eta;
  for (int j = 0; j <= N; ++j)
    for (int i = 0; i <= N - j; ++i, ++s) {
      const double cij = cij_of(i, j);
      double radial;  // (1-eta)^i P_i^{0,0}(2 csi/(1-eta) - 1)
      if (om == 0.0) radial = (i == 0) ? 1.0 : 0.0;
      else radial = std::pow(om, i) * jacobi(i, 0, 0, 2 * csi / om - 1);
      phi[s] = cij * std::pow(2.0, i) * radial * jacobi(j, 2 * i + 1, 0, 2 * eta - 1);
    }
}

void dubiner_grad(int N, double csi, double eta, double* gc, double* ge) {
  int s = 0;
  const double om = 1 - eta;
  for (int j = 0; j <= N; ++j)
    for (int i = 0; i <= N - j; ++i, ++s) {
      const double cij = cij_of(i, j);
      const double xx = 2 * csi / om - 1;
      if (i == 0 && j == 0) {
        gc[s] = 0;
        ge[s] = 0;
      } else if (i == 0) {
        gc[s] = 0;
        ge[s] = cij * (j + 2) * jacobi(j - 1, 2, 1, 2 * eta - 1);
      } else if (j == 0) {
        gc[s] = cij * std::pow(2.0, i) * std::pow(om, i - 1) * (i + 1) * jacobi(i - 1, 1, 1, xx);
        ge[s] = cij * std::pow(2.0, i) *
                (-i * std::pow(om, i - 1) * jacobi(i, 0, 0, xx) +
                 csi * std::pow(om, i - 2) * (i + 1) * jacobi(i - 1, 1, 1, xx));
      } else {
        const double pj = jacobi(j, 2 * i + 1, 0, 2 * eta - 1);
        gc[s] = cij * std::pow(2.0, i) * std::pow(om, i - 1) * (i + 1) * jacobi(i - 1, 1, 1, xx) * pj;
        ge[s] = cij * std::pow(2.0, i) *
                (-i * std::pow(om, i - 1) * jacobi(i, 0, 0, xx) * pj +
                 csi * std::pow(om, i - 2) * (i + 1) * jacobi(i - 1, 1, 1, xx) * pj +
                 std::pow(om, i) * (2 * i + j + 2) * jacobi(i, 0, 0, xx) * jacobi(j - 1, 2 * i + 2, 1, 2 * eta - 1));
      }
    }
}

// (1-eta)^(i-1) P^{1,1}_{i-1}(2 csi/(1-eta) - 1), a polynomial of degree i-1
// in (csi, eta); its value at the collapsed vertex (0, 1) is 1 for i = 1 and
// 0 above.
static double ba_radial(int i, double csi, double om) {
  if (om == 0.0) return i == 1 ? 1.0 : 0.0;
  return std::pow(om, i - 1) * jacobi(i - 1, 1, 1, 2 * csi / om - 1);
}

void ba_phi(int N, double csi, double eta, double* phi) {
  const double l0 = 1 - csi - eta, om = 1 - eta, yy = 2 * eta - 1;
  int s = 0;
  phi[s++] = l0;
  phi[s++] = csi;
  phi[s++] = eta;
  for (int i = 1; i < N; ++i) phi[s++] = l0 * csi * ba_radial(i, csi, om);
  for (int j = 1; j < N; ++j) phi[s++] = l0 * eta * jacobi(j - 1, 1, 1, yy);
  for (int j = 1; j < N; ++j) phi[s++] = csi * eta * jacobi(j - 1, 1, 1, yy);
  for (int j = 1; j < N; ++j)
    for (int i = 1; i + j < N; ++i) phi[s++] = l0 * csi * eta * ba_radial(i, csi, om) * jacobi(j - 1, 2 * i + 1, 1, yy);
}

void ba_grad(int N, double csi, double eta, double* gc, double* ge) {
  const double l0 = 1 - csi - eta, om = 1 - eta, yy = 2 * eta - 1, xx = 2 * csi / om - 1;
  int s = 0;
  gc[s] = -1; ge[s++] = -1;
  gc[s] = 1;  ge[s++] = 0;
  gc[s] = 0;  ge[s++] = 1;
  // Family A, l0 csi (1-eta)^(i-1) P^{1,1}_{i-1}(xx), using
  // d/dz P^{a,b}_n = (n + a + b + 1)/2 P^{a+1,b+1}_{n-1} and
  // dxx/dcsi = 2/(1-eta), dxx/deta = 2 csi/(1-eta)^2.
  for (int i = 1; i < N; ++i, ++s) {
    const double pa = jacobi(i - 1, 1, 1, xx), dp = jacobi(i - 2, 2, 2, xx);
    gc[s] = (1 - 2 * csi - eta) * std::pow(om, i - 1) * pa + l0 * csi * std::pow(om, i - 2) * dp * (i + 2);
    ge[s] = -std::pow(om, i - 2) * csi * (i + csi - i * csi - i * eta) * pa +
            csi * csi * l0 * std::pow(om, i - 3) * (i + 2) * dp;
  }
  // Family B, l0 eta P^{1,1}_{j-1}(2 eta - 1).
  for (int j = 1; j < N; ++j, ++s) {
    const double pj = jacobi(j - 1, 1, 1, yy);
    gc[s] = -eta * pj;
    ge[s] = (1 - csi - 2 * eta) * pj + l0 * eta * jacobi(j - 2, 2, 2, yy) * (j + 2);
  }
  // Family C, csi eta P^{1,1}_{j-1}(2 eta - 1).
  for (int j = 1; j < N; ++j, ++s) {
    const double pj = jacobi(j - 1, 1, 1, yy);
    gc[s] = eta * pj;
    ge[s] = csi * pj + eta * csi * (j + 2) * jacobi(j - 2, 2, 2, yy);
  }
  // Interior, l0 csi eta (1-eta)^(i-1) P^{1,1}_{i-1}(xx) P^{2i+1,1}_{j-1}(2 eta - 1).
  for (int j = 1; j < N; ++j)
    for (int i = 1; i + j < N; ++i, ++s) {
      const double pa = jacobi(i - 1, 1, 1, xx), dpa = jacobi(i - 2, 2, 2, xx);
      const double pb = jacobi(j - 1, 2 * i + 1, 1, yy), dpb = jacobi(j - 2, 2 * i + 2, 2, yy);
      gc[s] = eta * std::pow(om, i - 2) * pb * ((1 - 2 * csi - eta) * om * pa + l0 * csi * (i + 2) * dpa);
      ge[s] = csi * std::pow(om, i - 3) *
              ((om * om * (1 - csi - 2 * eta) - om * eta * l0 * (i - 1)) * pa * pb + csi * l0 * eta * (i + 2) * dpa * pb +
               l0 * eta * om * om * (j + 2 * i + 2) * pa * dpb);
    }
}

void basis_phi(int basis, int N, double csi, double eta, double* phi) {
  if (basis == kBoundaryAdapted) ba_phi(N, csi, eta, phi);
  else dubiner_phi(N, csi, eta, phi);
}

void basis_grad(int basis, int N, double csi, double eta, double* gc, double* ge) {
  if (basis == kBoundaryAdapted) ba_grad(N, csi, eta, gc, ge);
  else dubiner_grad(N, csi, eta, gc, ge);
}

bool spd_inverse(int n, const std::vector<double>& A, std::vector<double>* Ainv) {
  std::vector<double> L(size_t(n) * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = A[size_t(j) * n + j];
    for (int k = 0; k < j; ++k) d -= L[size_t(j) * n + k] * L[size_t(j) * n + k];
    if (!(d > 0)) return false;
    L[size_t(j) * n + j] = std::sqrt(d);
    for (int i = j + 1; i < n; ++i) {
      double v = A[size_t(i) * n + j];
      for (int k = 0; k < j; ++k) v -= L[size_t(i) * n + k] * L[size_t(j) * n + k];
      L[size_t(i) * n + j] = v / L[size_t(j) * n + j];
    }
  }
  // Columns of A^-1: solve L L^T x = e_c.
  Ainv->assign(size_t(n) * n, 0.0);
  std::vector<double> y(n);
  for (int c = 0; c < n; ++c) {
    for (int i = 0; i < n; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= L[size_t(i) * n + k] * y[k];
      y[i] = v / L[size_t(i) * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
      double v = y[i];
      for (int k = i + 1; k < n; ++k) v -= L[size_t(k) * n + i] * (*Ainv)[size_t(k) * n + c];
      (*Ainv)[size_t(i) * n + c] = v / L[size_t(i) * n + i];
    }
  }
  return true;
}

bool cholesky(int n, const std::vector<double>& A, std::vector<double>* L, std::vector<double>* Linv) {
  L->assign(size_t(n) * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = A[size_t(j) * n + j];
    for (int k = 0; k < j; ++k) d -= (*L)[size_t(j) * n + k] * (*L)[size_t(j) * n + k];
    if (!(d > 0)) return false;
    (*L)[size_t(j) * n + j] = std::sqrt(d);
    for (int i = j + 1; i < n; ++i) {
      double v = A[size_t(i) * n + j];
      for (int k = 0; k < j; ++k) v -= (*L)[size_t(i) * n + k] * (*L)[size_t(j) * n + k];
      (*L)[size_t(i) * n + j] = v / (*L)[size_t(j) * n + j];
    }
  }
  // L^-1 by forward substitution, column by column (lower triangular).
  Linv->assign(size_t(n) * n, 0.0);
  for (int c = 0; c < n; ++c)
    for (int i = c; i < n; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) v -= (*L)[size_t(i) * n + k] * (*Linv)[size_t(k) * n + c];
      (*Linv)[size_t(i) * n + c] = v / (*L)[size_t(i) * n + i];
    }
  return true;
}

static void edge_node(int l, double x, double* c, double* e) {
  // QuadratureRule_imp.hpp:66-91.
  if (l == 2) { *c = x; *e = 0.0; }
  else if (l == 0) { *c = 1.0 - x; *e = x; }
  else { *c = 0.0; *e = 1.0 - x; }
}

RefTables make_tables(int N, int basis) {
  RefTables T;
  T.N = N;
  T.basis = basis;
  T.Np = np_of(N);
  T.Q = N + 1;
  const int Np = T.Np, Q = T.Q;
  const size_t P2 = size_t(Np) * Np;
  std::vector<double> x1(Q), w1(Q), x(Q), w(Q);
  gauleg(Q, 0.0, 1.0, x1.data(), w1.data());
  gauleg(Q, -1.0, 1.0, x.data(), w.data());
  T.w1 = w1;
  // Volume: collapsed Gauss rule (QuadratureRule_imp.hpp:101-113).
  std::vector<double> gc(Np), ge(Np);
  T.K.assign(4 * P2, 0.0);
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j) {
      const double wq = (1 - x[i]) * w[i] * w[j] / 8.;
      const double c = (1 + x[i]) / 2., e = (1 - x[i]) * (1 + x[j]) / 4.;
      basis_grad(basis, N, c, e, gc.data(), ge.data());
      const double* g[2] = {gc.data(), ge.data()};
      for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
          for (int r = 0; r < Np; ++r)
            for (int s = 0; s < Np; ++s) T.K[(a * 2 + b) * P2 + size_t(r) * Np + s] += wq * g[a][r] * g[b][s];
    }
  // Edges.
  T.Be.assign(size_t(3) * Q * Np, 0.0);
  T.Ge.assign(size_t(3) * 2 * Q * Np, 0.0);
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < Q; ++k) {
      double c, e;
      edge_node(l, x1[k], &c, &e);
      basis_phi(basis, N, c, e, &T.Be[(size_t(l) * Q + k) * Np]);
      basis_grad(basis, N, c, e, &T.Ge[((size_t(l) * 2 + 0) * Q + k) * Np],
                 &T.Ge[((size_t(l) * 2 + 1) * Q + k) * Np]);
    }
  auto B = [&](int l, int k, int i) { return T.Be[(size_t(l) * Q + k) * Np + i]; };
  auto G = [&](int l, int a, int k, int i) { return T.Ge[((size_t(l) * 2 + a) * Q + k) * Np + i]; };
  T.Ws.assign(3 * P2, 0.0);
  T.Wx.assign(9 * P2, 0.0);
  T.Ds.assign(6 * P2, 0.0);
  T.Dx.assign(18 * P2, 0.0);
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < Q; ++k) {
      const int kk = Q - 1 - k;
      for (int i = 0; i < Np; ++i)
        for (int j = 0; j < Np; ++j) {
          T.Ws[l * P2 + size_t(i) * Np + j] += w1[k] * B(l, k, i) * B(l, k, j);
          for (int a = 0; a < 2; ++a) T.Ds[(a * 3 + l) * P2 + size_t(i) * Np + j] += w1[k] * G(l, a, k, i) * B(l, k, j);
          for (int lp = 0; lp < 3; ++lp) {
            T.Wx[(l * 3 + lp) * P2 + size_t(i) * Np + j] += w1[k] * B(l, k, i) * B(lp, kk, j);
            for (int a = 0; a < 2; ++a)
              T.Dx[((a * 3 + l) * 3 + lp) * P2 + size_t(i) * Np + j] += w1[k] * G(l, a, k, i) * B(lp, kk, j);
          }
        }
    }
  // Reference mass on the collapsed Gauss<N+1> rule: the integrand has degree
  // 2N, which the rule integrates exactly (the reference uses Dunavant<2N>
  // for BoundaryAdapted, equal up to rounding).
  T.Minv.assign(P2, 0.0);
  if (basis == kDubiner) {
    for (int i = 0; i < Np; ++i) T.Minv[size_t(i) * Np + i] = 1.0;
    T.M = T.Minv;
  } else {
    std::vector<double> M(P2, 0.0), ph(Np);
    for (int i = 0; i < Q; ++i)
      for (int j = 0; j < Q; ++j) {
        const double wq = (1 - x[i]) * w[i] * w[j] / 8.;
        basis_phi(basis, N, (1 + x[i]) / 2., (1 - x[i]) * (1 + x[j]) / 4., ph.data());
        for (int r = 0; r < Np; ++r)
          for (int c = 0; c < Np; ++c) M[size_t(r) * Np + c] += wq * ph[r] * ph[c];
      }
    spd_inverse(Np, M, &T.Minv);
    T.M = M;
  }
  return T;
}

Geometry make_geometry(int32_t ne, const double* xy, const int32_t* tri) {
  Geometry g;
  g.detJ.resize(ne);
  g.invJ.resize(size_t(ne) * 4);
  g.elen.resize(size_t(ne) * 3);
  g.enrm.resize(size_t(ne) * 6);
  static const int ends[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  for (int32_t e = 0; e < ne; ++e) {
    const double* p[3] = {xy + 2 * size_t(tri[3 * size_t(e)]), xy + 2 * size_t(tri[3 * size_t(e) + 1]),
                          xy + 2 * size_t(tri[3 * size_t(e) + 2])};
    // J = [p1 - p0 | p2 - p0] (Geometry.cpp:178-183), det and closed-form inverse.
    const double j00 = p[1][0] - p[0][0], j10 = p[1][1] - p[0][1];
    const double j01 = p[2][0] - p[0][0], j11 = p[2][1] - p[0][1];
    const double det = j00 * j11 - j10 * j01;
    const double invdet = 1.0 / det;
    g.detJ[e] = det;
    g.invJ[4 * size_t(e) + 0] = j11 * invdet;   // (0,0)
    g.invJ[4 * size_t(e) + 1] = -j10 * invdet;  // (1,0)
    g.invJ[4 * size_t(e) + 2] = -j01 * invdet;  // (0,1)
    g.invJ[4 * size_t(e) + 3] = j00 * invdet;   // (1,1)
    for (int l = 0; l < 3; ++l) {
      const double* a = p[ends[l][0]];
      const double* b = p[ends[l][1]];
      const double dx = a[0] - b[0], dy = a[1] - b[1];
      g.elen[3 * size_t(e) + l] = std::sqrt(dx * dx + dy * dy);
      const double nx = -a[1] + b[1], ny = a[0] - b[0];
      const double nn = std::sqrt(nx * nx + ny * ny);
      g.enrm[6 * size_t(e) + 2 * l + 0] = nx / nn;
      g.enrm[6 * size_t(e) + 2 * l + 1] = ny / nn;
    }
  }
  return g;
}

bool build_neighbours(int32_t ne, const int32_t* tri, int32_t* neigh, int32_t* nedge, std::string* err) {
  // Directed edge (a -> b) of face l; a neighbour owns the reversed edge.
  // The directed edges are bucketed by their first vertex (a CSR over the
  // vertices, a handful of edges per vertex), so finding the reversed edge
  // (b -> a) scans bucket b: O(ne) in all, no hashing.
  static const int ends[3][2] = {{1, 2}, {2, 0}, {0, 1}};
  int32_t nv = 0;
  for (size_t i = 0; i < size_t(ne) * 3; ++i) nv = std::max(nv, tri[i] + 1);
  std::vector<int32_t> start(size_t(nv) + 1, 0);
  for (size_t i = 0; i < size_t(ne) * 3; ++i) {
    const size_t e = i / 3;
    const int l = int(i % 3);
    start[size_t(tri[3 * e + ends[l][0]]) + 1]++;
  }
  for (int32_t v = 0; v < nv; ++v) start[size_t(v) + 1] += start[v];
  std::vector<int32_t> fill(start.begin(), start.end() - 1);
  std::vector<int32_t> to(size_t(ne) * 3), owner(size_t(ne) * 3);  // bucket entries: end vertex, element*3 + face
  for (int32_t e = 0; e < ne; ++e)
    for (int l = 0; l < 3; ++l) {
      const int32_t a = tri[3 * size_t(e) + ends[l][0]], b = tri[3 * size_t(e) + ends[l][1]];
      // The same directed edge twice: clockwise or overlapping triangles.
      for (int32_t q = start[a]; q < fill[a]; ++q)
        if (to[q] == b) {
          if (err) {
            std::ostringstream os;
            os << "directed edge (" << a << "," << b << ") shared by elements " << owner[q] / 3 << " and " << e
               << " (clockwise or overlapping triangles)";
            *err = os.str();
          }
          return false;
        }
      to[fill[a]] = b;
      owner[fill[a]] = 3 * e + l;
      ++fill[a];
    }
  for (int32_t e = 0; e < ne; ++e)
    for (int l = 0; l < 3; ++l) {
      const int32_t a = tri[3 * size_t(e) + ends[l][0]], b = tri[3 * size_t(e) + ends[l][1]];
      int32_t found = -1;
      for (int32_t q = start[b]; q < start[size_t(b) + 1]; ++q)
        if (to[q] == a) {
          found = owner[q];
          break;
        }
      if (found >= 0 && found / 3 != e) {
        neigh[3 * size_t(e) + l] = found / 3;
        nedge[3 * size_t(e) + l] = found % 3;
      } else {
        neigh[3 * size_t(e) + l] = -1;
        nedge[3 * size_t(e) + l] = -1;
      }
    }
  return true;
}

void bsr_pattern(int32_t ne, const int32_t* neigh, std::vector<int32_t>* row_ptr, std::vector<int32_t>* col,
                 std::vector<int8_t>* bface) {
  row_ptr->assign(size_t(ne) + 1, 0);
  col->clear();
  bface->clear();
  col->reserve(size_t(ne) * 4);
  bface->reserve(size_t(ne) * 4);
  for (int32_t e = 0; e < ne; ++e) {
    col->push_back(e);
    bface->push_back(-1);
    for (int l = 0; l < 3; ++l)
      if (neigh[3 * size_t(e) + l] >= 0) {
        col->push_back(neigh[3 * size_t(e) + l]);
        bface->push_back(int8_t(l));
      }
    (*row_ptr)[e + 1] = int32_t(col->size());
  }
}

namespace {

// Padded bounding box of element e. The pad covers every point the
// containment test below accepts: its tolerances are absolute in units of
// twice the area, i.e. a distance of about 1e-6 / (edge length) outside an
// edge, which the 1e-4 / (w + h) term bounds for any element size.
void element_box(const double* xy, const int32_t* tri, int32_t e, double box[4]) {
  const double* p0 = xy + 2 * size_t(tri[3 * size_t(e)]);
  const double* p1 = xy + 2 * size_t(tri[3 * size_t(e) + 1]);
  const double* p2 = xy + 2 * size_t(tri[3 * size_t(e) + 2]);
  const double xmin = std::fmin(p0[0], std::fmin(p1[0], p2[0])), xmax = std::fmax(p0[0], std::fmax(p1[0], p2[0]));
  const double ymin = std::fmin(p0[1], std::fmin(p1[1], p2[1])), ymax = std::fmax(p0[1], std::fmax(p1[1], p2[1]));
  const double wh = (xmax - xmin) + (ymax - ymin);
  const double pad = 1e-3 * wh + 1e-6 + (wh > 0 ? 1e-4 / wh : 0.0);
  box[0] = xmin - pad;
  box[1] = xmax + pad;
  box[2] = ymin - pad;
  box[3] = ymax + pad;
}

// Triangle::intriangle (Geometry.cpp:112-118) and invmap (Geometry.cpp:199-202)
// of element e; on success the basis values at the point go to phi.
bool try_element(int N, int basis, const double* xy, const int32_t* tri, const Geometry& g, int32_t e, double px,
                 double py, double* phi) {
  double box[4];
  element_box(xy, tri, e, box);
  if (px < box[0] || px > box[1] || py < box[2] || py > box[3]) return false;
  const double* p0 = xy + 2 * size_t(tri[3 * size_t(e)]);
  const double* p1 = xy + 2 * size_t(tri[3 * size_t(e) + 1]);
  const double* p2 = xy + 2 * size_t(tri[3 * size_t(e) + 2]);
  const double s = p0[1] * p2[0] - p0[0] * p2[1] + (p2[1] - p0[1]) * px + (p0[0] - p2[0]) * py;
  const double t = p0[0] * p1[1] - p0[1] * p1[0] + (p0[1] - p1[1]) * px + (p1[0] - p0[0]) * py;
  const double A = 1. / 2. * (-p1[1] * p2[0] + p0[1] * (-p1[0] + p2[0]) + p0[0] * (p1[1] - p2[1]) + p1[0] * p2[1]);
  if (!(s > -1e-6 && t > -1e-6 && (s + t) < (2 + 1e-6) * A)) return false;
  const double* iJ = &g.invJ[4 * size_t(e)];
  const double dx = px - p0[0], dy = py - p0[1];
  const double r0 = iJ[0] * dx + iJ[2] * dy;
  const double r1 = iJ[1] * dx + iJ[3] * dy;
  basis_phi(basis, N, r0, r1, phi);
  return true;
}

}  // namespace

int32_t locate_point(int N, int32_t ne, const double* xy, const int32_t* tri, const Geometry& g, double px,
                     double py, double* phi, int basis) {
  for (int32_t e = 0; e < ne; ++e)
    if (try_element(N, basis, xy, tri, g, e, px, py, phi)) return e;
  return -1;
}

void locate_points(int N, int32_t ne, const double* xy, const int32_t* tri, const Geometry& g, int32_t npts,
                   const double* pts, int32_t* elem, double* phi, int basis) {
  const int Np = np_of(N);
  if (npts <= 4) {
    for (int32_t k = 0; k < npts; ++k)
      elem[k] = locate_point(N, ne, xy, tri, g, pts[2 * k], pts[2 * k + 1], phi + size_t(k) * Np, basis);
    return;
  }
  // One pass over the elements in increasing id; the points (few against
  // the elements) are bucketed in a uniform grid, and each element tests
  // the points in the cells its padded box meets. A point takes the first
  // element that contains it: the same lowest-id element as a scan.
  double X0 = 1e300, X1 = -1e300, Y0 = 1e300, Y1 = -1e300;
  int32_t left = 0;
  for (int32_t k = 0; k < npts; ++k) {
    elem[k] = -1;
    const double px = pts[2 * k], py = pts[2 * k + 1];
    if (!(std::isfinite(px) && std::isfinite(py))) continue;
    X0 = std::fmin(X0, px);
    X1 = std::fmax(X1, px);
    Y0 = std::fmin(Y0, py);
    Y1 = std::fmax(Y1, py);
    ++left;
  }
  if (left == 0) return;
  const int G = std::max(1, std::min(1024, int(std::ceil(std::sqrt(double(left))))));
  const double W = std::fmax(X1 - X0, 1e-300), H = std::fmax(Y1 - Y0, 1e-300);
  auto cx = [&](double x) { return std::min(G - 1, std::max(0, int((x - X0) / W * G))); };
  auto cy = [&](double y) { return std::min(G - 1, std::max(0, int((y - Y0) / H * G))); };
  std::vector<int32_t> start(size_t(G) * G + 1, 0);
  std::vector<int32_t> list(static_cast<size_t>(left));
  for (int32_t k = 0; k < npts; ++k)
    if (std::isfinite(pts[2 * k]) && std::isfinite(pts[2 * k + 1]))
      start[size_t(cy(pts[2 * k + 1])) * G + cx(pts[2 * k]) + 1]++;
  for (size_t c = 0; c < size_t(G) * G; ++c) start[c + 1] += start[c];
  {
    std::vector<int32_t> fill(start.begin(), start.end() - 1);
    for (int32_t k = 0; k < npts; ++k)
      if (std::isfinite(pts[2 * k]) && std::isfinite(pts[2 * k + 1]))
        list[size_t(fill[size_t(cy(pts[2 * k + 1])) * G + cx(pts[2 * k])]++)] = k;
  }
  for (int32_t e = 0; e < ne && left > 0; ++e) {
    double b[4];
    element_box(xy, tri, e, b);
    if (b[1] < X0 || b[0] > X1 || b[3] < Y0 || b[2] > Y1) continue;  // meets no point
    for (int iy = cy(b[2]); iy <= cy(b[3]); ++iy)
      for (int ix = cx(b[0]); ix <= cx(b[1]); ++ix)
        for (int32_t i = start[size_t(iy) * G + ix]; i < start[size_t(iy) * G + ix + 1]; ++i) {
          const int32_t k = list[size_t(i)];
          const double px = pts[2 * k], py = pts[2 * k + 1];
          if (elem[k] >= 0 || px < b[0] || px > b[1] || py < b[2] || py > b[3]) continue;
          if (try_element(N, basis, xy, tri, g, e, px, py, phi + size_t(k) * Np)) {
            elem[k] = e;
            --left;
          }
        }
  }
}

bool gmsh_read(const std::string& path, std::vector<double>* xy, std::vector<int32_t>* tri,
               std::vector<int32_t>* region, std::string* err) {
  std::ifstream f(path);
  if (!f.is_open()) {
    *err = "Mesh file does not exist or is corrupted: " + path;
    return false;
  }
  std::string line;
  auto skip_to = [&](const char* tag) {
    while (std::getline(f, line))
      if (line.find(tag) != std::string::npos) return true;
    return false;
  };
  if (!skip_to("$Nodes")) {
    *err = "cannot find $Nodes in " + path;
    return false;
  }
  long nP = -1;
  if (!(f >> nP) || nP <= 0) {
    *err = "bad node count in " + path;
    return false;
  }
  xy->assign(size_t(nP) * 2, 0.0);
  std::unordered_map<long, int32_t> idmap;
  idmap.reserve(size_t(nP) * 2);
  for (long i = 0; i < nP; ++i) {
    long id;
    double x, y;
    if (!(f >> id >> x >> y)) {
      *err = "truncated $Nodes section in " + path;
      return false;
    }
    f.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
    (*xy)[2 * i] = x;
    (*xy)[2 * i + 1] = y;
    idmap[id] = int32_t(i);
  }
  if (!skip_to("$Elements")) {
    *err = "cannot find $Elements in " + path;
    return false;
  }
  long nE = -1;
  if (!(f >> nE) || nE < 0) {
    *err = "bad element count in " + path;
    return false;
  }
  tri->clear();
  region->clear();
  for (long i = 0; i < nE; ++i) {
    long id, type, ntags;
    if (!(f >> id >> type >> ntags)) {
      *err = "truncated $Elements section in " + path;
      return false;
    }
    std::vector<long> tags(size_t(ntags > 0 ? ntags : 0));
    for (auto& t : tags) f >> t;
    if (type == 2) {
      long a, b, c;
      f >> a >> b >> c;
      auto ia = idmap.find(a), ib = idmap.find(b), ic = idmap.find(c);
      if (ia == idmap.end() || ib == idmap.end() || ic == idmap.end()) {
        *err = "triangle refers to an unknown node in " + path;
        return false;
      }
      tri->push_back(ia->second);
      tri->push_back(ib->second);
      tri->push_back(ic->second);
      region->push_back(ntags >= 2 ? int32_t(tags[1]) : 0);  // elementary tag (Mesh.cpp:231)
    }
    f.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  }
  if (tri->empty()) {
    *err = "no triangles in " + path;
    return false;
  }
  return true;
}

void volume_rule(int N, std::vector<double>* c, std::vector<double>* e, std::vector<double>* w) {
  const int Q = N + 1;
  std::vector<double> x(Q), wx(Q);
  gauleg(Q, -1.0, 1.0, x.data(), wx.data());
  c->resize(size_t(Q) * Q);
  e->resize(size_t(Q) * Q);
  w->resize(size_t(Q) * Q);
  for (int i = 0; i < Q; ++i)
    for (int j = 0; j < Q; ++j) {
      (*w)[i * Q + j] = (1 - x[i]) * wx[i] * wx[j] / 8.;
      (*c)[i * Q + j] = (1 + x[i]) / 2.;
      (*e)[i * Q + j] = (1 - x[i]) * (1 + x[j]) / 4.;
    }
}

void quadrature_points(int N, int32_t ne, const double* xy, const int32_t* tri, double* pts) {
  std::vector<double> c, e, w;
  volume_rule(N, &c, &e, &w);
  const size_t nq = c.size();
  for (int32_t el = 0; el < ne; ++el) {
    const double* p0 = xy + 2 * size_t(tri[3 * size_t(el)]);
    const double* p1 = xy + 2 * size_t(tri[3 * size_t(el) + 1]);
    const double* p2 = xy + 2 * size_t(tri[3 * size_t(el) + 2]);
    for (size_t q = 0; q < nq; ++q) {
      // p0 + J x^, J = [p1 - p0 | p2 - p0]
      pts[(size_t(el) * nq + q) * 2 + 0] = p0[0] + ((p1[0] - p0[0]) * c[q] + (p2[0] - p0[0]) * e[q]);
      pts[(size_t(el) * nq + q) * 2 + 1] = p0[1] + ((p1[1] - p0[1]) * c[q] + (p2[1] - p0[1]) * e[q]);
    }
  }
}

void project(int N, int32_t ne, const double* xy, const int32_t* tri, const double* fvals, double* out, int basis) {
  std::vector<double> c, e, w;
  volume_rule(N, &c, &e, &w);
  const size_t nq = c.size();
  const int Np = np_of(N);
  std::vector<double> B(nq * Np);  // basis at the volume points, [q][i]
  for (size_t q = 0; q < nq; ++q) basis_phi(basis, N, c[q], e[q], &B[q * Np]);
  const RefTables T = make_tables(N, basis);
  const Geometry g = make_geometry(ne, xy, tri);
  std::vector<double> rhs(2 * size_t(Np));
  for (int32_t el = 0; el < ne; ++el) {
    std::fill(rhs.begin(), rhs.end(), 0.0);
    for (size_t q = 0; q < nq; ++q) {
      const double dx = std::abs(g.detJ[el]) * w[q];  // FESpace_imp.hpp:169
      const double* F = fvals + (size_t(el) * nq + q) * 2;
      for (int i = 0; i < Np; ++i) {
        rhs[i] += F[0] * dx * B[q * Np + i];
        rhs[Np + i] += F[1] * dx * B[q * Np + i];
      }
    }
    // uh = 1/detJ * M_ref^-1 * rhs (FESpace_imp.hpp:152-153); M_ref^-1 is the
    // identity for the orthonormal Dubiner basis (FESpace_imp.hpp:51-54).
    for (int i = 0; i < Np; ++i) {
      double a0 = 0.0, a1 = 0.0;
      for (int j = 0; j < Np; ++j) {
        a0 += T.Minv[size_t(i) * Np + j] * rhs[j];
        a1 += T.Minv[size_t(i) * Np + j] * rhs[Np + j];
      }
      out[size_t(el) * Np + i] = 1. / g.detJ[el] * a0;
      out[size_t(ne) * Np + size_t(el) * Np + i] = 1. / g.detJ[el] * a1;
    }
  }
}

void force_times(double dt, int64_t n, double* out) {
  if (n <= 0) return;
  out[0] = 0.0;
  double last = dt;
  for (int64_t k = 1; k < n; ++k) {
    const double t = last + dt;
    out[k] = t;
    last = t;
  }
}

double ricker(double t, double f0, double t0, double amp) {
  return amp * ((1 - 2 * M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)) *
                std::exp(-M_PI * M_PI * (f0 * f0) * (t - t0) * (t - t0)));
}

}  // namespace tsp
