// svf_layout.h - host-side direction-layout helpers (svf_layout.cpp).
#pragma once

#include <stdint.h>
#include <vector>

namespace svf
{

// (theta, phi) -> Cartesian direction and parabolic coordinates, as LoadBTF
// computes them.
void angles_to_cartesian(float theta, float phi, float* w);
void angles_to_parabolic(float theta, float phi, float* out);
// Euler angles of a quaternion's rotation as the reference obtains them
// (ToMatrix3, then Matrix3::decompose).
void quaternion_to_euler(const float* q, float* euler);
// ParabolicToCartesianCoordinates in the reference's operation order.
void parabolic_to_cartesian_ref(float px, float py, float* w);

uint32_t ring81_directions(float* lights_parabolic);
uint32_t fibonacci_directions(uint32_t count, float* lights_parabolic);

// Delaunay triangles (counter-clockwise) of the parabolic points; false when the
// result failed validation.
bool delaunay(const float* lights_parabolic, uint32_t n, std::vector<uint32_t>& triangles);

// Boundary edges in BTF::Edges order; returns the edge count.
uint32_t boundary_edges(const float* lights_parabolic, const std::vector<uint32_t>& triangles,
                        std::vector<uint32_t>& edges, std::vector<float>& angles);

// Layout-independent sample tables of the default initial guess, with the
// reference's float arithmetic.
struct InitHostTables
{
    float pdf;                            // 1 / (2 pi)
    double ndf_scale;                     // 1 / (4096 pdf)
    std::vector<float> ndf_dirs;          // [4096][3] NDF integrand light directions
    std::vector<int32_t> ndf_row_texel;   // NDF texels with n.z > 0
    std::vector<float> ndf_row_normal;    // [rows][3]
    std::vector<float> denom_w;           // [4096]
    std::vector<int32_t> pca_cell_id;     // [cells]
    std::vector<uint32_t> pca_cell_start; // [cells + 1]
    std::vector<uint32_t> pca_index;      // [262144] sample index, cell-grouped
    std::vector<float> pca_frac;          // [262144][2] cell-grouped
    std::vector<float> pca_dir;           // [262144][4] sample order
    std::vector<float> proj_dir;          // [1024][4]
    std::vector<float> proj_frac;         // [1024][2]
    std::vector<int32_t> proj_cell;       // [1024]
    float rot_s, rot_c;                   // tangent-plane rotation step
    int32_t axis_cell;                    // bilinear cell of (0, 0, 1)
    float axis_frac[2];
};

void build_init_host_tables(InitHostTables& tables);

// The directions DownsampleLightView keeps (svbrdf-lsq-fitting-setup.cc:129-163):
// n of L (2 <= n < L), one pseudo-randomly drawn per stride of (L - 1)/(n - 1).
// False when the draw cannot proceed (an empty stride).
bool downsample_light_view(uint32_t L, uint32_t n, uint32_t* idx);

} // namespace svf
