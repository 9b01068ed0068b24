// Host-side setup for the tspeed_b200 engine: reference element, mesh
// services and the factorised operator tables. Internal header.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tsp {

constexpr int kMaxN = 8;

// Modal bases of the reference (ShapeFunctions.hpp): Dubiner<N> is
// orthonormal, BoundaryAdapted<N> is not (its reference mass is dense).
enum Basis : int { kDubiner = 0, kBoundaryAdapted = 1 };

inline int np_of(int N) { return (N + 1) * (N + 2) / 2; }

// Gauss-Legendre nodes/weights on [a, b] by Newton iteration
// (QuadratureRule_imp.hpp:23-61).
void gauleg(int n, double a, double b, double* x, double* w);

// Jacobi polynomial P_n^{alpha,beta}(z) by the three-term recurrence of
// ShapeFunctions.cpp:25-60; zero for n < 0 as there.
double jacobi(int n, int alpha, int beta, double z);

// Dubiner basis values at (csi, eta), ShapeFunctions_imp.hpp:33-34, ordered
// j outer / i inner. At the collapsed vertex eta = 1 the reference formula is
// 0/0; the polynomial's limit is used there (the reference yields NaN).
void dubiner_phi(int N, double csi, double eta, double* phi);
// Reference gradients (d/dcsi, d/deta), ShapeFunctions_imp.hpp:35-50.
void dubiner_grad(int N, double csi, double eta, double* gcsi, double* geta);

// BoundaryAdapted basis values, ShapeFunctions_imp.hpp:55-118: the three
// vertex modes (1-csi-eta, csi, eta), N-1 edge modes on each of the edges
// eta = 0, csi = 0, csi + eta = 1, then the interior modes (j outer, i inner,
// i + j < N). At eta = 1 the polynomial's limit is used (the reference's
// formula is 0/0 there for degrees >= 3).
void ba_phi(int N, double csi, double eta, double* phi);
// Reference gradients of BoundaryAdapted<N>, eta < 1.
void ba_grad(int N, double csi, double eta, double* gcsi, double* geta);

void basis_phi(int basis, int N, double csi, double eta, double* phi);
void basis_grad(int basis, int N, double csi, double eta, double* gcsi, double* geta);

// Reference-element matrices of the factorised SIPG operator. All are
// Np x Np, row-major [i][j]; w = quadrature weights of Gauss<N+1>
// (QuadratureRule_imp.hpp:92-119), b_l(k) = basis on edge l at edge node k
// (edge parametrisation QuadratureRule_imp.hpp:66-91), g^a = reference
// gradient component a, kk = Q-1-k (the neighbour traverses the shared edge
// backwards, Matrices_imp.hpp:115,165).
//   K[a][b]    = sum_q w_q g^a_i g^b_j                 (volume)
//   Ws[l]      = sum_k w_k b_l(k)_i b_l(k)_j           (edge mass, self)
//   Wx[l][l']  = sum_k w_k b_l(k)_i b_l'(kk)_j         (edge mass, cross)
//   Ds[a][l]   = sum_k w_k g^a_l(k)_i b_l(k)_j         (traction trace, self)
//   Dx[a][l][l'] = sum_k w_k g^a_l(k)_i b_l'(kk)_j     (traction trace, cross)
struct RefTables {
  int N = 0, Np = 0, Q = 0, basis = kDubiner;
  // Inverse of the reference mass M_ij = sum_q w_q phi_i phi_j
  // (FESpace_imp.hpp:48-68): the identity for Dubiner, dense for
  // BoundaryAdapted. [Np][Np] row-major.
  std::vector<double> Minv;
  std::vector<double> M;   // the reference mass itself
  std::vector<double> K;   // [2][2][Np][Np]
  std::vector<double> Ws;  // [3][Np][Np]
  std::vector<double> Wx;  // [3][3][Np][Np]
  std::vector<double> Ds;  // [2][3][Np][Np]
  std::vector<double> Dx;  // [2][3][3][Np][Np]
  // Edge tabulation for the matrix-free kernel.
  std::vector<double> Be;  // [3][Q][Np]   basis on edge l at node k
  std::vector<double> Ge;  // [3][2][Q][Np] reference gradients on edges
  std::vector<double> w1;  // [Q]
};
RefTables make_tables(int N, int basis = kDubiner);

// Inverse of a symmetric positive definite n x n matrix (row-major) by
// Cholesky factorisation; false if a pivot is not positive.
bool spd_inverse(int n, const std::vector<double>& A, std::vector<double>* Ainv);
// A = L L^T (Cholesky, L lower triangular, row-major) and L^-1; false if A
// is not positive definite.
bool cholesky(int n, const std::vector<double>& A, std::vector<double>* L, std::vector<double>* Linv);

// Per-element geometry (Geometry.cpp:100-105, 125-132, 178-198): edge l is
// opposite vertex l with endpoints (1,2), (2,0), (0,1).
struct Geometry {
  std::vector<double> detJ;  // [ne] signed
  std::vector<double> invJ;  // [ne][4] (00, 10, 01, 11)  i.e. column-major 2x2
  std::vector<double> elen;  // [ne][3]
  std::vector<double> enrm;  // [ne][3][2]
};
Geometry make_geometry(int32_t ne, const double* xy, const int32_t* tri);

// O(ne) neighbour tables equal to Mesh::M_neighbors (Mesh.cpp:33-128) on
// conforming meshes. Returns false (with a message) on a repeated directed
// edge, i.e. a clockwise/overlapping triangle pair or a non-manifold edge.
bool build_neighbours(int32_t ne, const int32_t* tri, int32_t* neigh, int32_t* nedge, std::string* err);

// Block-CSR pattern of MyMat (MyMat.cpp:128-154); bface[b] = face of the row
// element shared with col[b], or -1 for the diagonal block.
void bsr_pattern(int32_t ne, const int32_t* neigh, std::vector<int32_t>* row_ptr, std::vector<int32_t>* col,
                 std::vector<int8_t>* bface);

// PointWiseEntity::M_add (Receivers_imp.hpp:34-51): the lowest-id element
// passing Triangle::intriangle (Geometry.cpp:112-118), reference coordinates
// by invmap (Geometry.cpp:199-202) and basis values. Returns -1 if none.
int32_t locate_point(int N, int32_t ne, const double* xy, const int32_t* tri, const Geometry& g, double px,
                     double py, double* phi, int basis = kDubiner);

// locate_point for many points with the same result: a uniform grid over the
// elements' padded bounding boxes gives each point its candidate elements in
// increasing id, and the first one passing the same test is taken.
// elem[k] = -1 where none does.
void locate_points(int N, int32_t ne, const double* xy, const int32_t* tri, const Geometry& g, int32_t npts,
                   const double* pts, int32_t* elem, double* phi, int basis = kDubiner);

// Gmsh 2.2 ASCII reader (Mesh.cpp:174-257).
bool gmsh_read(const std::string& path, std::vector<double>* xy, std::vector<int32_t>* tri,
               std::vector<int32_t>* region, std::string* err);

// The collapsed Gauss<N+1> volume rule on the reference triangle
// (QuadratureRule_imp.hpp:101-113): (N+1)^2 nodes (c, e) and weights w.
void volume_rule(int N, std::vector<double>* c, std::vector<double>* e, std::vector<double>* w);

// Reference points of FESpace::field_out / points_out (FESpace_imp.hpp:31-34).
constexpr double kFieldPoints[4][2] = {{0.2, 0.2}, {0.8, 0.2}, {0.2, 0.8}, {0.5, 0.5}};

// Physical volume quadrature points of every element, [ne][Q*Q][2], in the
// order of the collapsed Gauss<N+1> rule (QuadratureRule_imp.hpp:101-113)
// mapped by Triangle::map (Geometry.cpp:203-207).
void quadrature_points(int N, int32_t ne, const double* xy, const int32_t* tri, double* pts);

// FESpace::transform (FESpace_imp.hpp:136-179): L2 projection of a vector
// field given by its values at the quadrature points, fvals[ne][Q*Q][2], onto
// the modes of the basis, reference layout out[c*ne*Np + e*Np + i].
void project(int N, int32_t ne, const double* xy, const int32_t* tri, const double* fvals, double* out,
             int basis = kDubiner);

// Force evaluation times (TimeAdvance.cpp:28,46 with M_last_time
// accumulated in double, TimeAdvance.hpp:230).
void force_times(double dt, int64_t n, double* out);

// Ricker wavelet of Examples/src/Lamb.cpp:37 scaled by amp.
double ricker(double t, double f0, double t0, double amp);

}  // namespace tsp
