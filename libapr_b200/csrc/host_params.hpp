// Host-side parameter derivation for the GPU pipeline: recursive-filter
// coefficients, local-intensity-scale windows, level geometry and stencils.
//
// These are O(k0) / O(stencil) computations done once per call on the CPU,
// with the same libm functions and the same float/double evaluation order as
// the reference, so the GPU kernels receive bit-identical constants.
#pragma once

#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace aprb {

// Smoothing-spline recursive filter (ComputeGradient.hpp:256-330): b1, b2,
// norm_factor and the four boundary vectors folded to minLen taps.
struct IIRCoef {
    float b1 = 0, b2 = 0, norm = 1;
    int k0 = 0, minLen = 0;
    std::vector<float> bc1, bc2, bc3, bc4;  // minLen entries each (folded)
};
IIRCoef iir_coefficients(float lambda, int dim);

// get_window_alt (LocalIntensityScale.hpp:250-303)
struct LisWindow {
    int active[3] = {0, 0, 0};
    int win1[3] = {0, 0, 0};
    int win2[3] = {0, 0, 0};
    int n_active = 0;
    float rescale = 1;
};
LisWindow lis_window(const aprb_params &p, int yd, int xd, int zd);

// GenInfo::init (GenInfo.hpp:33-66) plus initialize_xz_linear offsets
// (LinearAccess.hpp:37-54).  Returns the xz_end length.
uint64_t apr_geometry(int y, int x, int z, Geom &g);
// GenInfo::init_tree (GenInfo.hpp:69-98)
uint64_t tree_geometry(int y, int x, int z, Geom &g);

// APRStencil::get_downsampled_stencils (APRStencil.hpp:13-95) for a cubic
// stencil of side ks: nlevels stencils packed back to back; sides[i] their side.
// T = float, or double for the FP64 instantiation of richardson_lucy.
template <typename T>
std::vector<T> downsampled_stencils(const T *stencil, int ks, int nlevels, bool normalize, std::vector<int> &sides);

}  // namespace aprb
