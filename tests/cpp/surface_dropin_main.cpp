// The reconstruction driver's calls (re.c:29, 107, 112-113) through the C++
// drop-in include/sphgpu_surface.hpp, with stand-ins for the reference's
// vec3d and vec3<INT_T>.  Reads n and n float positions, writes the field and
// the triangles.  Exit 3 with the library's message when a call fails.
#include <cstdio>
#include <cstdint>
#include <exception>
#include <vector>

#include "sphgpu_surface.hpp"

struct vec3d {
    double v[3] = {0, 0, 0};
    vec3d() = default;
    vec3d(double a, double b, double c) : v{a, b, c} {}
    double operator[](int i) const { return v[i]; }
};
struct vec3i {
    int v[3] = {0, 0, 0};
    vec3i() = default;
    vec3i(int a, int b, int c) : v{a, b, c} {}
    int operator[](int i) const { return v[i]; }
};

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int32_t n = 0;
    if (std::fread(&n, sizeof n, 1, f) != 1) return 2;
    std::vector<float> xyz(3 * (size_t)n);
    if (std::fread(xyz.data(), sizeof(float), xyz.size(), f) != xyz.size()) return 2;
    std::fclose(f);
    std::vector<vec3d> pos;
    double mn[3] = {1e30, 1e30, 1e30}, mx[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < n; ++i) {
        pos.emplace_back(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        for (int c = 0; c < 3; ++c) {
            mn[c] = pos.back()[c] < mn[c] ? pos.back()[c] : mn[c];
            mx[c] = pos.back()[c] > mx[c] ? pos.back()[c] : mx[c];
        }
    }
    try {
        sphgpu::surface_field<vec3d, vec3i> sf;
        sf.surface_setup(vec3d(mn[0], mn[1], mn[2]), vec3d(mx[0], mx[1], mx[2]), 0.01, 0.02, 0.005);
        const std::vector<float>& field = sf.surface_aniso(pos);
        std::vector<float> tris;
        const long long nt = sphgpu::marchingCubes(tris, 0.5f, sf);
        FILE* o = std::fopen(argv[2], "wb");
        const vec3i g = sf.get_grid_num();
        const int32_t hdr[3] = {g[0], g[1], g[2]};
        std::fwrite(hdr, sizeof hdr, 1, o);
        std::fwrite(field.data(), sizeof(float), field.size(), o);
        std::fclose(o);
        o = std::fopen(argv[3], "wb");
        std::fwrite(tris.data(), sizeof(float), 9 * (size_t)nt, o);
        std::fclose(o);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    return 0;
}
