// Shared definitions of the IFGF B200 library (host and device).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#ifdef __CUDACC__
#define IFGF_HD __host__ __device__ __forceinline__
#else
#define IFGF_HD inline
#endif

namespace ifgf
{

enum KernelKind : int
{
    K_LAPLACE = 0,
    K_HELMHOLTZ = 1,
    K_MODHELMHOLTZ = 2,
    K_GRADHELMHOLTZ = 3,
    K_DOUBLELAYER = 4,
    K_COMBINEDFIELD = 5,
    // wavenumber derivatives dG/dk of kernels 1 and 5 (no reference
    // counterpart; same tree, cones and orders as the base kernel)
    K_HELMHOLTZ_DK = 6,
    K_COMBINEDFIELD_DK = 7
};

enum Precision : int
{
    PREC_FP64 = 0,
    PREC_MIXED = 1
};

// Error carrying a C-ABI status code.
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

constexpr int MAX_LEVELS = 32;

// Geometry shared by every box of one source-tree level.  All boxes of a
// level have the same extent because children halve every dimension of the
// (non-cubic) root box (octree.hpp:1152-1163), so the side length H, the cone
// grids and the interpolation domain are per level.
struct LevelGeom
{
    double H;          // sideLength() of every box at this level
    double dmin[3];    // interpolation domain min: (smin, 0, -pi)
    double dmax[3];    // interpolation domain max: (smax, pi, pi)
    double hc[3];      // coarse (step 1) element widths
    double hf[3];      // fine (step 0) element widths
    double hci[3];     // 1 / hc
    double hfi[3];     // 1 / hf
    int nc[3];         // coarse cones per dimension
    int nf[3];         // fine cones per dimension
    int nbox;          // boxes at this level
    int box_off;       // first global box id of this level
    long long coarse_off; // first global coarse cone of this level
    long long n_coarse;   // active coarse cones at this level
    long long fine_off;   // first global fine cone of this level
    long long n_fine;     // active fine cones at this level
    long long fmap_off;   // offset of this level's dense fine map
    long long cmap_off;   // offset of this level's dense coarse map (setup only)
};

} // namespace ifgf
