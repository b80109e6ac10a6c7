// sphgpu_surface.hpp -- C++ drop-in for the reference's surface
// reconstruction: the class surface_field (surface_field.h:34-80) and
// marchingCubes (marching_cubes.h:16-17), as the reconstruction driver uses
// them (re.c:29, 107, 112-113), over the C ABI of sphgpu.h.
//
//   sphgpu::surface_field<vec3d, vec3<INT_T>> sf;          // was: surface_field sf;
//   sf.surface_setup(min, max, r_p, r_h, cell_size);
//   const std::vector<float>& f = sf.surface_aniso(positions);
//   std::vector<float> tris;                               // 9 floats per triangle
//   long long n = sphgpu::marchingCubes(tris, 0.5f, sf);   // the field stays on the GPU
//
// Vec3d is the caller's vector of three doubles (indexable with [], and
// constructible from three doubles), Vec3i its vector of three integers.
// Positions go to the GPU as floats.  Errors of the C ABI throw
// std::runtime_error with the library's message; particles outside the
// reconstruction box are left out of the field, as the reference's grid
// leaves them out (sphgpu_surface_field's SPHGPU_EOUT_OF_DOMAIN is not an
// error here; out_of_box() reports it).
#pragma once

#include <climits>
#include <stdexcept>
#include <string>
#include <vector>

#include "sphgpu.h"

namespace sphgpu {

inline void surface_check(sphgpu_surface_t h, long long rc, const char* what) {
    if (rc >= 0) return;
    char buf[256] = {0};
    if (h) sphgpu_surface_last_error(h, buf, (int)sizeof buf);
    throw std::runtime_error(std::string(what) + " failed (" + std::to_string(rc) + ")" + (buf[0] ? ": " : "") +
                             buf);
}

template <class Vec3d, class Vec3i>
class surface_field {
public:
    explicit surface_field(int device = 0) : device_(device) {}
    ~surface_field() {
        if (h_) sphgpu_surface_destroy(h_);
    }
    surface_field(const surface_field&) = delete;
    surface_field& operator=(const surface_field&) = delete;

    // surface_field::surface_setup (surface_field.cpp:8-41): the field grid
    // over [min, max] padded by the kernel radius, nodes cell_size apart
    void surface_setup(Vec3d min, Vec3d max, double r_p, double r_h, double cell_size) {
        if (h_) {
            sphgpu_surface_destroy(h_);
            h_ = nullptr;
        }
        const double mn[3] = {min[0], min[1], min[2]}, mx[3] = {max[0], max[1], max[2]};
        surface_check(nullptr, sphgpu_surface_create(mn, mx, r_p, r_h, cell_size, device_, &h_),
                      "sphgpu_surface_create");
        double gm[3], cell = 0;
        int num[3];
        surface_check(h_, sphgpu_surface_grid(h_, gm, num, &cell), "sphgpu_surface_grid");
        grid_min_ = Vec3d(gm[0], gm[1], gm[2]);
        grid_num_ = Vec3i(num[0], num[1], num[2]);
        cell_ = cell;
        field_.assign((size_t)num[0] * num[1] * num[2], 0.f);
    }

    // surface_field::surface_isotro (surface_field.cpp:43-75)
    const std::vector<float>& surface_isotro(const std::vector<Vec3d>& position) { return run(position, 0); }
    // surface_field::surface_aniso (surface_field.cpp:83-176)
    const std::vector<float>& surface_aniso(const std::vector<Vec3d>& position) { return run(position, 1); }

    const Vec3d& get_grid_min() const { return grid_min_; }
    const Vec3i& get_grid_num() const { return grid_num_; }
    double get_cell_size() const { return cell_; }
    const std::vector<float>& get_field() const { return field_; }

    // the library handle (the field stays on its GPU for marchingCubes)
    sphgpu_surface_t handle() const { return h_; }
    // particles the last field left out (outside the reconstruction box)
    bool out_of_box() const { return out_of_box_; }

private:
    const std::vector<float>& run(const std::vector<Vec3d>& position, int aniso) {
        if (!h_) throw std::runtime_error("surface_setup has not been called");
        if (position.size() > (size_t)INT_MAX) throw std::runtime_error("surface_field: more than INT_MAX particles");
        std::vector<float> xyz(3 * position.size());
        for (size_t i = 0; i < position.size(); ++i)
            for (int c = 0; c < 3; ++c) xyz[3 * i + c] = (float)position[i][c];
        const int rc = sphgpu_surface_field(h_, aniso, xyz.data(), (int)position.size(), 0);
        out_of_box_ = rc == SPHGPU_EOUT_OF_DOMAIN;
        if (!out_of_box_) surface_check(h_, rc, "sphgpu_surface_field");
        surface_check(h_, sphgpu_surface_get_field(h_, field_.data()), "sphgpu_surface_get_field");
        return field_;
    }

    int device_;
    sphgpu_surface_t h_ = nullptr;
    Vec3d grid_min_{};
    Vec3i grid_num_{};
    double cell_ = 0;
    std::vector<float> field_;
    bool out_of_box_ = false;
};

// marchingCubes (marching_cubes.cpp:45-120) over the field the surface_field
// holds on its GPU, the grid being its own (get_grid_min, get_grid_num,
// get_cell_size): result receives 9 floats per triangle in cube order (z,
// y, x), the count is returned.  ref_rows = 1 pairs the cube rows as the
// reference's row caches do (see sphgpu_surface_mesh).
template <class Vec3d, class Vec3i>
long long marchingCubes(std::vector<float>& result, float iso, const surface_field<Vec3d, Vec3i>& sf,
                        int ref_rows = 0) {
    sphgpu_surface_t h = sf.handle();
    if (!h) throw std::runtime_error("surface_setup has not been called");
    const long long n = sphgpu_surface_mesh(h, iso, ref_rows, nullptr, 0);
    surface_check(h, n, "sphgpu_surface_mesh");
    result.resize(9 * (size_t)n);
    const long long m = sphgpu_surface_mesh(h, iso, ref_rows, result.data(), n);
    surface_check(h, m, "sphgpu_surface_mesh");
    return m;
}

}  // namespace sphgpu
