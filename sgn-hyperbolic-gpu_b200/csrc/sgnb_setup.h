// sgnb_setup.h -- host-side set-up: FR tables, node coordinates, bathymetry statics.
#pragma once

#include <vector>

namespace sgnb {

// FROperators1D (src/core/fr_operators.h:57-115), degree P <= 7: Gauss-Lobatto points,
// or Gauss-Legendre points (gauss; fr_operators.cpp:86-100).
struct FrTables {
  int P = 0;
  bool gauss = false;
  double nodes[8] = {}, D[64] = {}, lL[8] = {}, lR[8] = {}, gLp[8] = {}, gRp[8] = {}, qw[8] = {};
};

// CartesianMesh2D geometry (src/core/mesh2d.h:23-51).
struct Mesh {
  int Nx = 0, Ny = 0;
  double Lx = 0, Ly = 0, hx = 0, hy = 0;
  int ex0 = 0;  // global index of the first element column (slabs of a larger mesh)
  // the slab's right edge is the periodic wrap of the larger mesh: the depth across it is
  // sampled at x = 0, where the whole mesh samples the first column's left faces
  bool wrapx = false;
};

// Bathymetry statics read by the kernels (SGN2D accessors, src/solver/sgn2d.h:94-98),
// plus the depth on the right / top domain edges used by walls.
struct Bathymetry {
  std::vector<double> Hnod, Hx, Hy, HfX, HfY, HfXEnd, HfYEnd;
};

bool fr_tables(int P, FrTables& t, bool gauss = false);
double still_depth(int kind, const double* p, double x, double y);
// number of doubles a parameter vector of this kind must hold (-1: unknown kind)
int bathy_param_count(int kind, const double* p, int n);
void node_coords(const Mesh& m, const FrTables& t, double* x, double* y);
void bathymetry(const Mesh& m, const FrTables& t, int kind, const double* p, Bathymetry& out);
// Nodal dH/dx, dH/dy: the element-local GLL derivative of the nodal depth over the
// Jacobian (src/solver/sgn2d.cpp:54-71); the fused kernels form the same values from the
// depth tile instead of reading them.
void depth_gradients(const Mesh& m, const FrTables& t, const double* Hnod, double* Hx,
                     double* Hy);
// Transpose of bathymetry() for kind 5 (cell means p = {Mx, My, Lx, Ly, means...}):
// cotangents of every static (bar) -> cotangent of the Mx * My means.
void cells_transpose(const Mesh& m, const FrTables& t, const double* p, const Bathymetry& bar,
                     double* means_bar);

}  // namespace sgnb
