// Scalar and container types of the RCWA API (rcwa/defns.h:7-23 of the
// reference), backed by Eigen when it is available and by a minimal shim
// otherwise.
#pragma once
#include <complex>
#include <vector>

typedef double scalar;
typedef std::complex<scalar> scalex;

#if defined(RCWA_B200_USE_EIGEN) || (defined(__has_include) && __has_include(<Eigen/Core>) && !defined(RCWA_B200_NO_EIGEN))
#include <Eigen/Core>
namespace Eigen {
typedef Eigen::Matrix<scalar, Eigen::Dynamic, 1> VectorXs;
typedef Eigen::Matrix<scalar, Eigen::Dynamic, Eigen::Dynamic> MatrixXs;
typedef Eigen::Matrix<scalex, Eigen::Dynamic, 1> VectorXcs;
typedef Eigen::Matrix<scalex, Eigen::Dynamic, Eigen::Dynamic> MatrixXcs;
}  // namespace Eigen
#else
#include "eigen_shim.h"
#endif

constexpr scalar Pi = 3.1415926535897932;

enum FieldComponent { Ex = 0, Ey = 1, Ez = 2, Hx = 3, Hy = 4, Hz = 5 };
enum SliceType { sliceXY = 0, sliceXZ = 1, sliceYZ = 2 };
enum SaveOption { modulation = 0, realpart = 1, imagpart = 2 };
