// Fields inside a solved stack: the mode amplitudes of every interior layer
// (RCWASolver::evaluateIntermediateField, rcwa/RCWASolver.cpp:1505-1644) and
// one field component on a slice as RCWASolver::saveFieldImage evaluates it
// (rcwa/RCWASolver.cpp:707-1012, no layer translation).
#pragma once
#include <vector>

#include "common.cuh"

// One solved point of a plan: device pointers into the plan's workspace.
struct FieldPoint {
  int N = 0, nx = 0, ny = 0, L = 0;
  std::vector<const cplx*> W, V, gamma;  // per stack layer (n x n, n x n, n)
  std::vector<const cplx*> Einv;         // per stack layer: permittivity ContinuousXY inverse (interior only)
  std::vector<double> thick;             // per stack layer
  const cplx* Rud = nullptr;             // n x n, the point's solved S-matrix blocks
  const cplx* Tdd = nullptr;
  const cplx* ab = nullptr;              // alpha[N] then beta[N]
  bool pat0 = false;                     // the incidence half-space is patterned
  double k0 = 0.0, kx0 = 0.0, ky0 = 0.0;
  double x0 = 0.0, y0 = 0.0, Lx = 0.0, Ly = 0.0;  // cell-grid origin and periods
};

// Rows of the slice for nres1 columns (saveFieldImage's nRes2).
int field_rows(const FieldPoint& fp, int slice, int nres1);

// The field (nres2 x nres1 complex, host memory) of component 0..5 (Ex, Ey,
// Ez, Hx, Hy, Hz) on slice 0 (XY at depth coord), 1 (XZ at y = coord) or 2
// (YZ at x = coord), depth measured from the top of the first interior
// layer, for the incident plane wave (px, py) of generateHorizontalPlaneWave.
// Allocates its device buffers (about 7 n^2 complex per interface) and
// synchronises st.  Returns an RCWA status.
int field_slice(const FieldPoint& fp, cplx px, cplx py, int slice, double coord, int component, int nres1,
                cplx* out, cudaStream_t st);
