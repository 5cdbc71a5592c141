// Host geometry: binary STL, the heightmap voxeliser of the reference's
// GeometryEngine (06_transient_localization_dx1.cpp:60-193) and a seeded
// synthetic city generator.  Built with -ffp-contract=off: every FP64
// expression of the ray cast keeps the reference's operation order so the
// voxelised mask is bit-identical.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

struct lbm_city_params;

namespace lbm {

class HeightField
{
public:
    // GeometryEngine::load (06:70-111) from memory: 9 floats per triangle,
    // vertex * scale + offset in FP64.
    void set_triangles(const float* tris, int ntris, double scale, double sx, double sy, double sz);
    // GeometryEngine::load (06:70-111) from a binary STL file: kStlNotOpened
    // (geometry left empty) when the file cannot be opened, kStlTruncated
    // when it ends before the triangle count of its header (the missing
    // records read as zeros, as in the reference), else kStlLoaded.
    static constexpr int kStlLoaded = 0, kStlNotOpened = 1, kStlTruncated = 2;
    int load_stl(const std::string& path, double scale, double sx, double sy, double sz);
    // GeometryEngine::getGroundHeight (06:144-192): highest hit of the ray
    // from z = 10000 straight down, -1e30 when there is none.
    double ground_height(double x, double y) const;
    size_t triangle_count() const { return tris_.size(); }
    // The bin grid and triangles as flat arrays for the device ray cast
    // (voxel.cu): tri15 = per triangle v1, v2, v3, min, max (15 doubles).
    void export_flat(std::vector<double>& tri15, std::vector<int>& bin_start, std::vector<int>& bin_items,
                     double gmin[3], double gmax[3], double& cell_w, double& cell_h) const;

private:
    struct Tri
    {
        double v1[3], v2[3], v3[3], mn[3], mx[3];
    };
    void build_bins();   // GeometryEngine::buildGrid (06:113-142), 200 x 200 bins

    std::vector<Tri> tris_;
    double gmin_[3] = {1e30, 1e30, 1e30};
    double gmax_[3] = {-1e30, -1e30, -1e30};
    double cell_w_ = 1.0, cell_h_ = 1.0;
    std::vector<int> bin_start_;   // CSR offsets, 200*200+1
    std::vector<int> bin_items_;
};

// Seeded city of axis-aligned box buildings on a street grid; 12 triangles
// per box, vertices on multiples of dx.  Returns the plan coverage reached.
double city_generate(const lbm_city_params& p, std::vector<float>& tris);
bool stl_write(const char* path, const float* tris, int ntris);

// HeightField::ground_height of every column of the halo-inclusive grid on
// the GPU, bit-identical to the host: gH[j * nxt + i] for the cell centre
// x = x_min + (i - 0.5) dx, y = y_min + (j - 0.5) dx (voxel.cu).
int ground_height_device(const HeightField& geo, double x_min, double y_min, double dx, int nxt, int nyt,
                         double* gH, void* stream);

}  // namespace lbm
