#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>

#include "nlos_lbm.h"

namespace lbm {

namespace {
constexpr int kBinRows = 200, kBinCols = 200;   // GeometryEngine::gridRows/gridCols (06:66)
}

void HeightField::set_triangles(const float* v, int ntris, double scale, double sx, double sy, double sz)
{
    tris_.assign((size_t)std::max(ntris, 0), Tri{});
    for (int d = 0; d < 3; ++d)
    {
        gmin_[d] = 1e30;
        gmax_[d] = -1e30;
    }
    const double off[3] = {sx, sy, sz};
    for (int i = 0; i < ntris; ++i)
    {
        const float* p = v + 9 * (size_t)i;
        Tri& t = tris_[i];
        for (int d = 0; d < 3; ++d)
        {
            t.v1[d] = p[d] * scale + off[d];
            t.v2[d] = p[3 + d] * scale + off[d];
            t.v3[d] = p[6 + d] * scale + off[d];
            t.mn[d] = std::min({t.v1[d], t.v2[d], t.v3[d]});
            t.mx[d] = std::max({t.v1[d], t.v2[d], t.v3[d]});
            gmin_[d] = std::min(gmin_[d], t.mn[d]);
            gmax_[d] = std::max(gmax_[d], t.mx[d]);
        }
    }
    build_bins();
}

int HeightField::load_stl(const std::string& path, double scale, double sx, double sy, double sz)
{
    std::ifstream file(path, std::ios::binary);
    if (!file)
    {
        set_triangles(nullptr, 0, scale, sx, sy, sz);
        return kStlNotOpened;
    }
    file.seekg(0, std::ios::end);
    const long long size = (long long)file.tellg();
    file.seekg(0, std::ios::beg);
    char header[80];
    file.read(header, 80);
    uint32_t n = 0;
    file.read(reinterpret_cast<char*>(&n), 4);
    if (!file) n = 0;
    // The reference reads n records whatever the file holds; a short read
    // leaves a record's missing bytes zero (its StlTriangle st{}, 06:82-85).
    // Records past the end of the file are all-zero triangles: degenerate at
    // the offset point, they never hit a ray and add only that point to the
    // bounding box, so one of them stands for all (the mask is the same, and
    // a corrupt count cannot make this allocate more than the file holds).
    const long long avail = size > 84 ? (size - 84 + 49) / 50 : 0;   // records with at least one byte
    const bool truncated = (long long)n > (size > 84 ? (size - 84) / 50 : 0);
    const long long kept = std::min<long long>(n, avail) + ((long long)n > avail ? 1 : 0);
    std::vector<float> v((size_t)kept * 9, 0.0f);
    for (long long i = 0; i < std::min<long long>(n, avail); ++i)
    {
        unsigned char rec[50] = {0};
        file.read(reinterpret_cast<char*>(rec), 50);
        std::memcpy(&v[(size_t)i * 9], rec + 12, 36);
    }
    set_triangles(v.data(), (int)kept, scale, sx, sy, sz);
    return truncated ? kStlTruncated : kStlLoaded;
}

void HeightField::build_bins()
{
    bin_start_.clear();
    bin_items_.clear();
    if (tris_.empty()) return;
    cell_w_ = (gmax_[0] - gmin_[0]) / kBinRows;
    cell_h_ = (gmax_[1] - gmin_[1]) / kBinCols;
    if (cell_w_ < 1e-9) cell_w_ = 1.0;
    if (cell_h_ < 1e-9) cell_h_ = 1.0;
    std::vector<int> span(tris_.size() * 4);
    bin_start_.assign((size_t)kBinRows * kBinCols + 1, 0);
    auto clampi = [](int v, int hi) { return std::max(0, std::min(hi, v)); };
    for (size_t i = 0; i < tris_.size(); ++i)
    {
        const Tri& t = tris_[i];
        int r1 = clampi((int)((t.mn[0] - gmin_[0]) / cell_w_), kBinRows - 1);
        int r2 = clampi((int)((t.mx[0] - gmin_[0]) / cell_w_), kBinRows - 1);
        int c1 = clampi((int)((t.mn[1] - gmin_[1]) / cell_h_), kBinCols - 1);
        int c2 = clampi((int)((t.mx[1] - gmin_[1]) / cell_h_), kBinCols - 1);
        span[4 * i] = r1; span[4 * i + 1] = r2; span[4 * i + 2] = c1; span[4 * i + 3] = c2;
        for (int r = r1; r <= r2; ++r)
            for (int c = c1; c <= c2; ++c) bin_start_[(size_t)r * kBinCols + c + 1]++;
    }
    for (size_t b = 0; b < (size_t)kBinRows * kBinCols; ++b) bin_start_[b + 1] += bin_start_[b];
    bin_items_.resize((size_t)bin_start_.back());
    std::vector<int> fill((size_t)kBinRows * kBinCols, 0);
    for (size_t i = 0; i < tris_.size(); ++i)
        for (int r = span[4 * i]; r <= span[4 * i + 1]; ++r)
            for (int c = span[4 * i + 2]; c <= span[4 * i + 3]; ++c)
            {
                const size_t b = (size_t)r * kBinCols + c;
                bin_items_[(size_t)bin_start_[b] + fill[b]++] = (int)i;
            }
}

double HeightField::ground_height(double x, double y) const
{
    if (tris_.empty()) return -1e30;
    if (x < gmin_[0] || x > gmax_[0] || y < gmin_[1] || y > gmax_[1]) return -1e30;
    const int r = (int)((x - gmin_[0]) / cell_w_);
    const int c = (int)((y - gmin_[1]) / cell_h_);
    if (r < 0 || r >= kBinRows || c < 0 || c >= kBinCols) return -1e30;
    const size_t b = (size_t)r * kBinCols + c;
    if (bin_start_[b] == bin_start_[b + 1]) return -1e30;

    // Moller-Trumbore, ray origin (x, y, 10000), direction (0, 0, -1), EPS 1e-9.
    const double ro[3] = {x, y, 10000.0};
    const double rd[3] = {0.0, 0.0, -1.0};
    const double EPS = 1e-9;
    double max_z = -1e30;
    for (int n = bin_start_[b]; n < bin_start_[b + 1]; ++n)
    {
        const Tri& t = tris_[bin_items_[n]];
        if (t.mx[0] < x - 1e-6 || t.mn[0] > x + 1e-6) continue;
        if (t.mx[1] < y - 1e-6 || t.mn[1] > y + 1e-6) continue;
        const double e1[3] = {t.v2[0] - t.v1[0], t.v2[1] - t.v1[1], t.v2[2] - t.v1[2]};
        const double e2[3] = {t.v3[0] - t.v1[0], t.v3[1] - t.v1[1], t.v3[2] - t.v1[2]};
        const double h[3] = {rd[1] * e2[2] - rd[2] * e2[1], rd[2] * e2[0] - rd[0] * e2[2], rd[0] * e2[1] - rd[1] * e2[0]};
        const double a = e1[0] * h[0] + e1[1] * h[1] + e1[2] * h[2];
        if (std::abs(a) < EPS) continue;
        const double f = 1.0 / a;
        const double s[3] = {ro[0] - t.v1[0], ro[1] - t.v1[1], ro[2] - t.v1[2]};
        const double u = f * (s[0] * h[0] + s[1] * h[1] + s[2] * h[2]);
        if (u < 0.0 || u > 1.0) continue;
        const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
        const double v = f * (rd[0] * q[0] + rd[1] * q[1] + rd[2] * q[2]);
        if (v < 0.0 || (u + v) > 1.0) continue;
        const double tt = f * (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]);
        if (tt > EPS)
        {
            const double hit = ro[2] + tt * rd[2];
            if (hit > max_z) max_z = hit;
        }
    }
    return max_z;
}

void HeightField::export_flat(std::vector<double>& tri15, std::vector<int>& bin_start, std::vector<int>& bin_items,
                              double gmin[3], double gmax[3], double& cell_w, double& cell_h) const
{
    tri15.resize(tris_.size() * 15);
    for (size_t i = 0; i < tris_.size(); ++i)
        for (int d = 0; d < 3; ++d)
        {
            tri15[15 * i + d] = tris_[i].v1[d];
            tri15[15 * i + 3 + d] = tris_[i].v2[d];
            tri15[15 * i + 6 + d] = tris_[i].v3[d];
            tri15[15 * i + 9 + d] = tris_[i].mn[d];
            tri15[15 * i + 12 + d] = tris_[i].mx[d];
        }
    bin_start = bin_start_;
    bin_items = bin_items_;
    for (int d = 0; d < 3; ++d)
    {
        gmin[d] = gmin_[d];
        gmax[d] = gmax_[d];
    }
    cell_w = cell_w_;
    cell_h = cell_h_;
}

// ---------------------------------------------------------------- city

namespace {

struct SplitMix64
{
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    int uniform(int lo, int hi)   // inclusive
    {
        if (hi <= lo) return lo;
        return lo + (int)(next() % (uint64_t)(hi - lo + 1));
    }
};

// Street-grid partition of [margin, n - margin) into block spans of
// footprint size in [fp_min, fp_max] separated by gaps of at least `street`.
std::vector<std::pair<int, int>> spans(SplitMix64& rng, int n, const lbm_city_params& p)
{
    std::vector<std::pair<int, int>> out;
    int x = p.margin;
    const int end = n - p.margin;
    while (x + p.fp_min <= end)
    {
        int w = rng.uniform(p.fp_min, p.fp_max);
        if (x + w > end) w = end - x;
        if (w < p.fp_min) break;
        out.push_back({x, x + w});
        x += w + p.street + rng.uniform(0, p.street / 2);
    }
    return out;
}

void push_box(std::vector<float>& t, double x0, double y0, double z0, double x1, double y1, double z1)
{
    const double v[8][3] = {{x0, y0, z0}, {x1, y0, z0}, {x1, y1, z0}, {x0, y1, z0},
                            {x0, y0, z1}, {x1, y0, z1}, {x1, y1, z1}, {x0, y1, z1}};
    // Outward-facing quads, each split along its first diagonal.
    const int quads[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};
    for (const auto& qd : quads)
    {
        const int tri[2][3] = {{qd[0], qd[1], qd[2]}, {qd[0], qd[2], qd[3]}};
        for (const auto& tr : tri)
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) t.push_back((float)v[tr[c]][d]);
    }
}

}  // namespace

double city_generate(const lbm_city_params& p, std::vector<float>& tris)
{
    tris.clear();
    SplitMix64 rng{p.seed};
    const auto xs = spans(rng, p.nx, p);
    const auto ys = spans(rng, p.ny, p);
    std::vector<std::pair<int, int>> blocks;
    for (int a = 0; a < (int)xs.size(); ++a)
        for (int b = 0; b < (int)ys.size(); ++b) blocks.push_back({a, b});
    for (int i = (int)blocks.size() - 1; i > 0; --i) std::swap(blocks[i], blocks[rng.uniform(0, i)]);
    const double total = (double)p.nx * (double)p.ny;
    double covered = 0.0;
    for (const auto& blk : blocks)
    {
        if (covered / total >= p.coverage) break;
        const auto& sx = xs[blk.first];
        const auto& sy = ys[blk.second];
        const int h = rng.uniform(p.h_min, p.h_max);
        push_box(tris, sx.first * p.dx, sy.first * p.dx, 0.0, sx.second * p.dx, sy.second * p.dx, h * p.dx);
        covered += (double)(sx.second - sx.first) * (double)(sy.second - sy.first);
    }
    return covered / total;
}

bool stl_write(const char* path, const float* tris, int ntris)
{
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return false;
    char header[80] = {0};
    std::snprintf(header, sizeof header, "nlos_lbm synthetic geometry");
    bool ok = std::fwrite(header, 1, 80, fp) == 80;
    const uint32_t n = (uint32_t)ntris;
    ok = ok && std::fwrite(&n, 4, 1, fp) == 1;
    for (int i = 0; ok && i < ntris; ++i)
    {
        const float* v = tris + 9 * (size_t)i;
        const double a[3] = {(double)v[3] - v[0], (double)v[4] - v[1], (double)v[5] - v[2]};
        const double b[3] = {(double)v[6] - v[0], (double)v[7] - v[1], (double)v[8] - v[2]};
        double nrm[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const double len = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        unsigned char rec[50] = {0};
        float nf[3] = {0.f, 0.f, 0.f};
        if (len > 0)
            for (int d = 0; d < 3; ++d) nf[d] = (float)(nrm[d] / len);
        std::memcpy(rec, nf, 12);
        std::memcpy(rec + 12, v, 36);
        ok = std::fwrite(rec, 1, 50, fp) == 50;
    }
    return std::fclose(fp) == 0 && ok;
}

}  // namespace lbm
