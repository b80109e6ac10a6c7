/* C entry points around the reference's surface reconstruction (test
 * infrastructure, built by oracle/build_ref.py into
 * oracle/_ref/libref_surface.so): surface_field (surface_field.cpp, with the
 * TNT / JAMA stand-in of jama_svd.h) and marchingCubes (marching_cubes.cpp),
 * as the reference's own driver re.c:29,107,112-113 calls them.
 *
 * The reference's ker_spline and weight_wij keep their constants in
 * function-local statics set on the first call (surface_field.cpp:237-241,
 * 255), so every surface_field in one process uses the radii of the first
 * one that computed a field. */
#include <cstring>
#include <vector>

#include "marching_cubes.h"
#include "surface_field.h"

extern "C" {
void* rsf_create(const double* mn, const double* mx, double r_p, double r_h, double cell) {
    surface_field* s = new surface_field();
    s->surface_setup(vec3d(mn[0], mn[1], mn[2]), vec3d(mx[0], mx[1], mx[2]), r_p, r_h, cell);
    return s;
}
void rsf_destroy(void* h) { delete static_cast<surface_field*>(h); }
void rsf_grid(void* h, double* mn, int* num, double* cell) {
    surface_field* s = static_cast<surface_field*>(h);
    for (int i = 0; i < 3; ++i) { mn[i] = s->get_grid_min()[i]; num[i] = (int)s->get_grid_num()[i]; }
    *cell = s->get_cell_size();
}
/* field of n positions (3 doubles each); aniso: surface_aniso, else
 * surface_isotro; returns the node count */
long long rsf_field(void* h, int aniso, const double* xyz, int n, float* out) {
    surface_field* s = static_cast<surface_field*>(h);
    std::vector<vec3d> p(n);
    for (int i = 0; i < n; ++i) p[i] = vec3d(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    const std::vector<float>& f = aniso ? s->surface_aniso(p) : s->surface_isotro(p);
    if (out) memcpy(out, f.data(), sizeof(float) * f.size());
    return (long long)f.size();
}
/* marchingCubes over a field (x fastest, then y, then z); triangles of 9
 * floats into out (capacity max_tris); returns the triangle count */
long long rsf_marching_cubes(float iso, const float* field, const float* mn, const int* res, float cell, float* out,
                             long long max_tris) {
    std::vector<float> grid(field, field + (size_t)res[0] * res[1] * res[2]);
    std::vector<float> result;
    const int_t n = marchingCubes(result, iso, grid, vec3f(mn[0], mn[1], mn[2]), veci_t(res[0], res[1], res[2]), cell);
    if (out) memcpy(out, result.data(), sizeof(float) * 9 * (size_t)(n < max_tris ? n : max_tris));
    return (long long)n;
}
}
